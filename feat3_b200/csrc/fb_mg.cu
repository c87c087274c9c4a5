// Native multigrid driver: device hierarchy (SELL-C-sigma level matrices, CSR transfers,
// Dirichlet bit masks), the fused V-cycle, PCG / Richardson outer solvers in FP64 and in
// mixed precision (FP64 outer defect and update around an FP32 V-cycle with FP32 or FP16
// matrix values), structured Q1/Q2 device assembly, and the adjoint gradient.
//
// The operator sequence is the reference's (kernel/solver/multigrid.hpp:1268-2000,
// pcg.hpp:188-287, richardson.hpp:160-226, jacobi_precond.hpp:137-165); fusion only merges
// operations that the reference performs back to back on the same rows:
//   * pre-smoothing from a zero guess: step 1 is an element-wise Jacobi update (fused into
//     the restriction that produced the level's right-hand side), steps 2..nu are fused
//     defect+update SpMVs; the smoother's final defect equals the defect multigrid
//     recomputes afterwards, so it is computed once;
//   * post-smoothing: Richardson on the correction from zero with rhs d = b - A s0 equals
//     Jacobi on the level system started at s0 (same iterates in exact arithmetic), so each
//     step is one fused SpMV and the discarded last smoother defect is never formed;
//   * the smoother's initial-norm test (skip on a non-finite or <= eps^2 defect) is kept:
//     the norm is reduced inside the kernel that produces the defect and read by the next.
#include "fb_mg_internal.cuh"
#include "fb_mf.cuh"
#include "fb_mf_stream.cuh"
#include "fb_stencil_stream.cuh"
#include "fb_rest_staged.cuh"
#include "fb_coarse.cuh"

#include <algorithm>
#include <cstdio>
#include <initializer_list>
#include <cstring>
#include <numeric>
#include <vector>

#undef FB_CHECK_LAUNCH
#define FB_CHECK_LAUNCH()                                                              \
  do {                                                                                 \
    cudaError_t _e = cudaGetLastError();                                               \
    if (_e == cudaSuccess && fb::debug_enabled()) _e = fb::debug_sync(m->stream, __FILE__, __LINE__); \
    if (_e != cudaSuccess) return FB_ERR_CUDA;                                         \
  } while (0)

namespace fb {

static int occupancy_grid(const void* fn, uint64_t work_warps) {
  // blocks of 256 threads; at most the resident capacity of all SMs
  int bps = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, fn, 256, 0) != cudaSuccess || bps < 1) bps = 4;
  uint64_t need = (work_warps + 7) / 8;
  uint64_t cap = uint64_t(bps) * kSMs;
  uint64_t g = need < cap ? need : cap;
  return int(g < 1 ? 1 : g);
}

// launch with the programmatic-dependent-launch attribute (the kernel begins with pdl_wait())
template<typename... KArgs, typename... Args>
static cudaError_t launch_pdl(cudaStream_t s, void (*fn)(KArgs...), dim3 grid, dim3 block, size_t smem, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute at;
  at.id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at.val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = &at;
  cfg.numAttrs = pdl_enabled() ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, fn, static_cast<KArgs>(args)...);
}

// ------------------------------------------------------------------ launch helpers
// debugging aid (FB_DEBUG=1): report pointers that are not device memory of this context
static void debug_check_ptrs(const char* what, std::initializer_list<const void*> ptrs) {
  int i = 0;
  for (const void* p : ptrs) {
    cudaPointerAttributes at;
    cudaError_t e = cudaPointerGetAttributes(&at, p);
    if (p && (e != cudaSuccess || at.type != cudaMemoryTypeDevice))
      std::fprintf(stderr, "feat3_b200: %s pointer #%d = %p is not device memory (err %d type %d)\n", what, i, p,
                   int(e), e == cudaSuccess ? int(at.type) : -1);
    cudaGetLastError();
    ++i;
  }
}

template<typename VT, typename XT, typename AT, typename Epi>
static int launch_sell(fb_mg* m, const DevSell& A, int prec, const XT* x, const Epi& epi, double* red_out) {
  // 2-byte values are read two slots per load from their interleaved layout (k_quant16_sell): 534
  // against 579 us per FP16 Jacobi step at 257^3 with one 2-byte load per slot and 32 slots in
  // flight per lane (602 us with 16, 624 us with 8); unrolling the pair loop 2 or 4 times ran 814-817
  // us. Their odd last slot, if any, takes the slot loop below the pair loop.
  auto fn = k_sell<VT, XT, AT, Epi, 8>;
  const int grid = occupancy_grid((const void*)fn, A.nchunks);
  if (debug_enabled())
    debug_check_ptrs("k_sell", {A.cs, A.cl, A.col, A.view(prec).val, (const void*)x, (const void*)m->ws,
                                (const void*)m->counter, (const void*)red_out, (const void*)A.perm});
  fn<<<grid, 256, 0, m->stream>>>(A.view(prec), x, epi, m->ws, m->counter, red_out);
  m->launches++;
  FB_CHECK_LAUNCH();
  return FB_OK;
}

template<typename VT, typename XT, typename AT, typename Epi>
static int launch_csr(fb_mg* m, const DevCsr& A, bool f32, const XT* x, const Epi& epi, double* red_out) {
  const double avg = A.rows ? double(A.nnz) / double(A.rows) : 0.0;
  if (avg <= 4.0) {
    auto fn = k_csr_epi<VT, XT, AT, Epi, 4>;
    fn<<<occupancy_grid((const void*)fn, (uint64_t(A.rows) * 4 + 31) / 32), 256, 0, m->stream>>>(A.view(f32), x, epi, m->ws, m->counter, red_out);
  } else if (avg <= 12.0) {
    auto fn = k_csr_epi<VT, XT, AT, Epi, 8>;
    fn<<<occupancy_grid((const void*)fn, (uint64_t(A.rows) * 8 + 31) / 32), 256, 0, m->stream>>>(A.view(f32), x, epi, m->ws, m->counter, red_out);
  } else {
    auto fn = k_csr_epi<VT, XT, AT, Epi, 16>;
    fn<<<occupancy_grid((const void*)fn, (uint64_t(A.rows) * 16 + 31) / 32), 256, 0, m->stream>>>(A.view(f32), x, epi, m->ws, m->counter, red_out);
  }
  m->launches++;
  FB_CHECK_LAUNCH();
  return FB_OK;
}

template<typename VT, typename XT, typename AT, typename Epi, int S>
static int launch_stencil_S(fb_mg* m, const DevStencil& St, const void* val, float scale, uint32_t rows,
                            const XT* x, const Epi& epi, double* red_out) {
  StencilView<S> v;
  v.rows = rows; v.nchunks = St.nchunks; v.val = val; v.scale = scale;
  for (int j = 0; j < S; ++j) v.off[j] = St.off[j];
  constexpr int G = S == 27 ? 9 : S;
  auto fn = k_stencil<VT, XT, AT, Epi, S, G>;
  fn<<<occupancy_grid((const void*)fn, St.nchunks), 256, 0, m->stream>>>(v, x, epi, m->ws, m->counter, red_out);
  m->launches++;
  FB_CHECK_LAUNCH();
  return FB_OK;
}

// the stored offsets are those of a lattice of M1 points per side (lattice_off)
template<int S, int CM1>
static bool offsets_are(const DevStencil& St, uint32_t M1) {
  if (M1 != uint32_t(CM1)) return false;
  for (int j = 0; j < S; ++j)
    if (St.off[j] != lattice_off<S, CM1>(j)) return false;
  return true;
}

// levels of 257^3 and 129^3 points take the lattice size as a compile-time constant
template<typename VT, typename Epi, int S>
static int launch_stencil_packed_S(fb_mg* m, const DevStencil& St, const void* val, float scale, uint32_t rows,
                                   uint32_t M1, const float* x, const Epi& epi, double* red_out) {
  StencilView<S> v;
  v.rows = rows; v.nchunks = St.nchunks; v.val = val; v.scale = scale;
  for (int j = 0; j < S; ++j) v.off[j] = St.off[j];
  auto fn = k_stencil_packed<VT, Epi, S>;
  if constexpr (S == 27) {
    if (offsets_are<S, 257>(St, M1)) fn = k_stencil_packed<VT, Epi, S, 257>;
    else if (offsets_are<S, 129>(St, M1)) fn = k_stencil_packed<VT, Epi, S, 129>;
  }
  fn<<<occupancy_grid((const void*)fn, St.nchunks), 256, 0, m->stream>>>(v, x, epi, m->ws, m->counter, red_out);
  m->launches++;
  FB_CHECK_LAUNCH();
  return FB_OK;
}

// the streaming stencil SpMV on the 257^3 level (x staged once per run, register window): one CTA
// of 16 consumer warps per SM (slabs of two planes), 4 stages of 6 lines (FP16 values)
template<typename VT, typename Epi>
static int launch_stencil_stream(fb_mg* m, const void* val, float scale, const float* x, const Epi& epi,
                                 double* red_out) {
  using SE = Staged<Epi>;
  constexpr int NS = SE::kStreams, NCW = 16, TY = 6, NST = 4, NT = 32 * (NCW + 1);
  constexpr uint32_t M1 = 257, W = M1 - 2;
  auto r16 = [](uint64_t b) { return uint32_t((b + 15) & ~uint64_t(15)); };
  StStream G{};
  G.G = std::max<uint32_t>(1, uint32_t(32 * NCW) / W);
  G.nslab = (W + G.G - 1) / G.G;
  G.units = uint64_t(G.nslab) * W;
  G.cap_x = r16(uint64_t(TY) * M1 * sizeof(float)) + 32;
  G.cap_s = NS ? r16(uint64_t(TY) * M1 * sizeof(float)) + 32 : 0;
  G.stage_bytes = ((G.G + 2) * G.cap_x + NS * G.G * G.cap_s + 127) & ~127u;
  G.nbl_items = (4 * M1 - 4) * ((M1 + 31) / 32);
  G.nedge_items = (W * W + 15) / 16;
  G.scale = scale;
  G.inject = m->inject;
  const size_t dyn = size_t(NST) * G.stage_bytes;
  auto fn = k_stencil_stream<VT, Epi, NST, TY, 257, NCW>;
  static size_t attr = 0;  // per instantiation: largest dynamic shared memory requested so far
  if (dyn > attr) {
    FB_CUDA(cudaFuncSetAttribute((const void*)fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(dyn)));
    attr = dyn;
  }
  int bps = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, (const void*)fn, NT, dyn) != cudaSuccess || bps < 1) {
    cudaGetLastError();
    bps = 1;
  }
  const uint32_t grid = uint32_t(std::min<uint64_t>(G.units, uint64_t(bps) * kSMs));
  const float* s0 = NS > 0 ? static_cast<const float*>(SE::stream(epi, 0)) : nullptr;
  const float* s1 = NS > 1 ? static_cast<const float*>(SE::stream(epi, 1)) : nullptr;
  FB_CUDA(launch_pdl(m->stream, fn, dim3(grid), dim3(NT), dyn, G, static_cast<const VT*>(val), x, epi, s0, s1, m->ws,
                     m->counter, red_out, m->kerr));
  m->launches++;
  FB_CHECK_LAUNCH();
  return FB_OK;
}

template<typename VT, typename XT, typename AT, typename Epi>
static int launch_stencil(fb_mg* m, const Level& L, int prec, const XT* x, const Epi& epi, double* red_out) {
  const DevStencil& St = L.St;
  if constexpr (!std::is_same<VT, double>::value) {
    // 2- and 4-byte values use the packed layout (8-byte loads per lane)
    const float scale = prec == FB_PREC_F16 ? St.scale16 : 1.0f;
    const void* pv = prec == FB_PREC_F16 ? (const void*)St.v16 : (const void*)St.v32;
    if constexpr (Staged<Epi>::kOk && std::is_same<XT, float>::value && std::is_same<VT, __half>::value) {
      // FP16 values at 257^3 with the lattice boundary as the filter: the streaming form (246
      // against 294 us per Jacobi step, FP16-stencil mixed solve 43.5 against 46.8 ms; with FP32
      // values, 14 value loads per row, it ran slower: 396 against 364 us)
      if (St.S == 27 && offsets_are<27, 257>(St, L.M1) && L.mask_boundary && L.mask &&
          Staged<Epi>::mask(epi) == L.mask && Staged<Epi>::input_is_x(epi, x) && !(m->cfg.flags & FB_FLAG_NO_STREAM))
        return launch_stencil_stream<VT, Epi>(m, pv, scale, x, epi, red_out);
    }
    if (St.S == 27) return launch_stencil_packed_S<VT, Epi, 27>(m, St, pv, scale, L.n, L.M1, x, epi, red_out);
    if (St.S == 9) return launch_stencil_packed_S<VT, Epi, 9>(m, St, pv, scale, L.n, L.M1, x, epi, red_out);
    return FB_ERR_UNSUPPORTED;
  }
  const void* val = prec == FB_PREC_F64 ? (const void*)St.v64 : (prec == FB_PREC_F32 ? (const void*)St.v32 : (const void*)St.v16);
  const float scale = prec == FB_PREC_F16 ? St.scale16 : 1.0f;
  if (St.S == 27) return launch_stencil_S<VT, XT, AT, Epi, 27>(m, St, val, scale, L.n, x, epi, red_out);
  if (St.S == 9) return launch_stencil_S<VT, XT, AT, Epi, 9>(m, St, val, scale, L.n, x, epi, red_out);
  return FB_ERR_UNSUPPORTED;
}

// ------------------------------------------------------------------ small kernels
// s1 = skip ? 0 : omega * filter_cor(invd o b)   (first pre-smoothing step from zero)
template<typename T>
__global__ void k_jacobi0(T* out, const T* __restrict__ b, const T* __restrict__ invd, const uint32_t* mask,
                          const double* skip_src, T omega, uint32_t n) {
  const bool skip = smoother_skip<T>(skip_src);
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    out[i] = (skip || masked(mask, i)) ? T(0) : omega * (invd[i] * b[i]);
}

// post-smoothing with nu == 1: restore the prolongated iterate when the smoother skipped
template<typename T>
__global__ void k_skip_fix(T* out, const T* __restrict__ s0, const double* skip_src, uint32_t n) {
  if (!smoother_skip<T>(skip_src)) return;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) out[i] = s0[i];
}

// dense coarse solve: x = Cinv b (Cinv = inverse of the filtered coarse matrix, zero
// Dirichlet rows/columns); one warp per row
template<typename T>
__global__ void k_dense_solve(T* x, const T* __restrict__ cinv, const T* __restrict__ b, uint32_t n) {
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= n) return;
  double s = 0.0;
  for (uint32_t j = lane; j < n; j += 32) s += double(cinv[uint64_t(warp) * n + j]) * double(b[j]);
  s = warp_sum(s);
  if (lane == 0) x[warp] = T(s);
}

// coarse "none": x = filter_cor(b)
template<typename T>
__global__ void k_copy_masked(T* x, const T* __restrict__ b, const uint32_t* mask, uint32_t n) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    x[i] = masked(mask, i) ? T(0) : b[i];
}

// Unpreconditioned CG on the coarsest level in one CTA, with the reference's default settings
// (Solver::new_pcg(matrix, filter), used as coarse solver by tutorial_05_multigrid.cpp:420-436):
// x = 0, r = b, stop on tol_rel = sqrt(eps) relative to ||r0||, divergence, non-finite
// defects or max_iter = 100 (pcg.hpp:139-287, iterative.hpp:216-235, 744-832).
template<typename T, int THREADS>
__global__ void __launch_bounds__(THREADS) k_coarse_cg(CsrView A, const T* __restrict__ b, T* x, T* r, T* p, T* q,
                                                        const uint32_t* mask, uint32_t n, int max_iter) {
  __shared__ double sh[THREADS / 32];
  __shared__ double bc;
  const T* val = static_cast<const T*>(A.val);
  auto dot = [&](const T* u, const T* v) -> double {
    double a = 0.0;
    for (uint32_t i = threadIdx.x; i < n; i += THREADS) a += double(u[i]) * double(v[i]);
    __syncthreads();
    const double s = block_sum<THREADS>(a, sh);
    if (threadIdx.x == 0) bc = s;
    __syncthreads();
    return bc;
  };
  const double e = double(eps_of<T>());
  const double tol_rel = sqrt(e), div_rel = 1.0 / e, big = 1.0 / (e * e);
  for (uint32_t i = threadIdx.x; i < n; i += THREADS) { r[i] = b[i]; x[i] = T(0); }
  __syncthreads();
  const double d0 = sqrt(dot(r, r));
  if (!isfinite(d0) || d0 <= e * e) return;
  for (uint32_t i = threadIdx.x; i < n; i += THREADS) p[i] = masked(mask, i) ? T(0) : r[i];
  __syncthreads();
  double gamma = dot(r, p);
  for (int it = 1; it <= max_iter; ++it) {
    for (uint32_t i = threadIdx.x; i < n; i += THREADS) {
      T s = T(0);
      for (uint32_t k = A.rp[i]; k < A.rp[i + 1]; ++k) s += val[k] * p[A.col[k]];
      q[i] = masked(mask, i) ? T(0) : s;
    }
    __syncthreads();
    const T alpha = T(gamma / dot(q, p));
    const bool upd = fabs(double(alpha)) >= e;
    for (uint32_t i = threadIdx.x; i < n; i += THREADS) {
      if (upd) { x[i] = alpha * p[i] + x[i]; r[i] = (-alpha) * q[i] + r[i]; }
    }
    __syncthreads();
    const double dc = sqrt(dot(r, r));
    if (!isfinite(dc) || dc > big || dc > div_rel * d0) return;
    if (dc <= big && dc <= tol_rel * d0) return;
    for (uint32_t i = threadIdx.x; i < n; i += THREADS) q[i] = masked(mask, i) ? T(0) : r[i];  // z
    __syncthreads();
    const double g2 = gamma;
    gamma = dot(r, q);
    const T beta = T(gamma / g2);
    const bool ub = fabs(double(beta)) >= e;
    for (uint32_t i = threadIdx.x; i < n; i += THREADS) p[i] = ub ? beta * p[i] + q[i] : q[i];
    __syncthreads();
  }
}

// PCG update: alpha = rz / qp; x += alpha p; r -= alpha q; ||r||^2 (+ FP32 copy of r)
// (pcg.hpp:241-251 with the |alpha| < eps shortcut of dense_vector.hpp:891-895)
// When s1 != nullptr the kernel also forms the first pre-smoothing step of the next V-cycle
// from zero, s1 = omega * filter_cor(invd o r) in the V-cycle's type (k_jacobi0 on the new r;
// the smoother's skip test is not needed there: the next V-cycle runs only after the host
// has found ||r|| finite and above the tolerance, and a skipped smoother with nu >= 2 is
// restored by the second step, which sees the same skip test).
template<typename T> struct Pair;
template<> struct Pair<float> { using type = float2; };
template<> struct Pair<double> { using type = double2; };

template<bool LOW>
// The x update x += alpha p of this step is deferred to a later k_pcg_dir2, which reads p
// anyway (or to k_pcg_finish2 after the last iteration): the same operation on the same values,
// fewer passes over p and x. Two rows per thread and
// step, with 8- and 16-byte accesses (all vectors are allocation bases, so pairs are aligned).
__global__ void __launch_bounds__(256) k_pcg_update(double* r, float* r32, const double* __restrict__ q,
                                                    DevScalars* sc, uint32_t n, double* ws, unsigned* counter,
                                                    double* rr_out, void* s1, const void* invd, const uint32_t* mask,
                                                    double omega) {
  using T = typename std::conditional<LOW, float, double>::type;
  using T2 = typename Pair<T>::type;
  pdl_wait();
  __shared__ double sh[8];
  // alpha = gamma' / (q . p) with gamma' = r . z of this iteration (pcg.hpp:241-251); the thread
  // that finishes the reduction then commits gamma <- gamma' for the next direction update
  const double alpha = sc->rz / sc->qp;
  const bool upd = fabs(alpha) >= eps_of<double>();
  T* s1t = static_cast<T*>(s1);
  const T* invt = static_cast<const T*>(invd);
  const T om = T(omega);
  double acc = 0.0;
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
  for (uint32_t j = tid; j < n / 2; j += stride) {
    const uint32_t i = 2 * j;
    double2 rv = reinterpret_cast<const double2*>(r)[j];
    if (upd) {
      const double2 qv = __ldg(reinterpret_cast<const double2*>(q) + j);
      rv.x = (-alpha) * qv.x + rv.x;
      rv.y = (-alpha) * qv.y + rv.y;
      reinterpret_cast<double2*>(r)[j] = rv;
    }
    if (LOW) reinterpret_cast<float2*>(r32)[j] = make_float2(float(rv.x), float(rv.y));
    if (s1t) {
      const uint32_t w = mask ? __ldg(mask + (i >> 5)) : 0u;  // i even: rows i, i+1 share the word
      const T2 iv = reinterpret_cast<const T2*>(invt)[j];
      T2 o;
      o.x = ((w >> (i & 31)) & 1u) ? T(0) : om * (iv.x * T(rv.x));
      o.y = ((w >> ((i + 1) & 31)) & 1u) ? T(0) : om * (iv.y * T(rv.y));
      reinterpret_cast<T2*>(s1t)[j] = o;
    }
    acc += rv.x * rv.x;
    acc += rv.y * rv.y;
  }
  if ((n & 1u) && tid == 0) {  // the last row of an odd count
    const uint32_t i = n - 1;
    double ri = r[i];
    if (upd) {
      ri = (-alpha) * q[i] + ri;
      r[i] = ri;
    }
    if (LOW) r32[i] = float(ri);
    if (s1t) s1t[i] = masked(mask, i) ? T(0) : om * (invt[i] * T(ri));
    acc += ri * ri;
  }
  pdl_trigger();
  const double blk = block_sum<256>(acc, sh);
  if (reduce_finish<256>(blk, ws, counter, rr_out, sh, false)) {
    sc->gamma = sc->rz;
    sc->alpha = upd ? alpha : 0.0;
  }
}

// r . z with z in FP64 or FP32 (ConvertPrecond: z = double(z_inner))
template<typename ZT>
__global__ void __launch_bounds__(256) k_dot_rz(const double* __restrict__ r, const ZT* __restrict__ z, uint32_t n,
                                                double* ws, unsigned* counter, double* out) {
  pdl_wait();
  __shared__ double sh[8];
  double acc = 0.0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    acc += r[i] * double(z[i]);
  pdl_trigger();
  const double blk = block_sum<256>(acc, sh);
  reduce_finish<256>(blk, ws, counter, out, sh, false);
}

// p = z + beta p, beta = rz / gamma (pcg.hpp:275-282); gamma <- rz is committed by k_pcg_update.
// PT = float: the direction is stored rounded to FP32 (the mixed matrix-free form); q = A p,
// x += alpha p and q . p then all use the stored direction, so r stays the defect of x, and only
// the conjugacy of successive directions carries the FP32 rounding, below that of the FP32
// preconditioner. The pending x updates (pcg.hpp:256) are deferred over two iterations:
// iteration j writes p_j into the buffer j & 1 (pout), from p_{j-1} in the other one (pin). An even
// j (HOLD) does not touch x: it holds alpha_{j-1} (sc->alpha_hold), whose direction p_{j-1} stays
// in pin. An odd j applies both pending steps in their order, x += alpha_{j-2} p_{j-2} (held, read
// from pout before it is overwritten), then x += alpha_{j-1} p_{j-1}: the x updates of PCG on the
// same values in the same order, with one read and one write of x per two iterations.
template<typename ZT, typename PT, bool HOLD>
__global__ void k_pcg_dir2(PT* pout, const PT* __restrict__ pin, double* x, const ZT* __restrict__ z, DevScalars* sc,
                           uint32_t n) {
  using P2 = typename Pair<PT>::type;
  using Z2 = typename Pair<ZT>::type;
  pdl_wait();
  const double beta = sc->rz / sc->gamma;
  const bool upd = fabs(beta) >= eps_of<double>();
  const double a1 = HOLD ? 0.0 : sc->alpha_hold, a2 = HOLD ? 0.0 : sc->alpha;
  const bool x1 = a1 != 0.0, x2 = a2 != 0.0;
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
  for (uint32_t j = tid; j < n / 2; j += stride) {
    const P2 pv = reinterpret_cast<const P2*>(pin)[j];
    const Z2 zv = __ldg(reinterpret_cast<const Z2*>(z) + j);
    const double p0 = double(pv.x), p1 = double(pv.y);
    if (!HOLD && (x1 || x2)) {
      double2 xv = reinterpret_cast<const double2*>(x)[j];
      if (x1) {
        const P2 hv = reinterpret_cast<const P2*>(pout)[j];
        xv.x = a1 * double(hv.x) + xv.x;
        xv.y = a1 * double(hv.y) + xv.y;
      }
      if (x2) {
        xv.x = a2 * p0 + xv.x;
        xv.y = a2 * p1 + xv.y;
      }
      reinterpret_cast<double2*>(x)[j] = xv;
    }
    P2 o;
    o.x = PT(upd ? beta * p0 + double(zv.x) : double(zv.x));
    o.y = PT(upd ? beta * p1 + double(zv.y) : double(zv.y));
    reinterpret_cast<P2*>(pout)[j] = o;
  }
  if ((n & 1u) && tid == 0) {
    const uint32_t i = n - 1;
    const double pi = double(pin[i]);
    if (!HOLD && (x1 || x2)) {
      double xi = x[i];
      if (x1) xi = a1 * double(pout[i]) + xi;
      if (x2) xi = a2 * pi + xi;
      x[i] = xi;
    }
    pout[i] = PT(upd ? beta * pi + double(z[i]) : double(z[i]));
  }
  if (HOLD && tid == 0) sc->alpha_hold = sc->alpha;
}

// the x updates still pending after the last iteration J (pcg.hpp:256): alpha_{J-1} p_{J-1}
// (held, J even) and alpha_J p_J, in that order
template<typename PT>
__global__ void k_pcg_finish2(double* x, const PT* __restrict__ phold, const PT* __restrict__ plast,
                              const DevScalars* sc, uint32_t n, int use_hold) {
  const double a1 = use_hold ? sc->alpha_hold : 0.0, a2 = sc->alpha;
  if (a1 == 0.0 && a2 == 0.0) return;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double xi = x[i];
    if (a1 != 0.0) xi = a1 * double(phold[i]) + xi;
    if (a2 != 0.0) xi = a2 * double(plast[i]) + xi;
    x[i] = xi;
  }
}

__global__ void k_init_pcg(DevScalars* sc) {
  sc->gamma = 1.0;
  sc->rz = 0.0;
  sc->alpha = 0.0;
  sc->alpha_hold = 0.0;
}

// adaptive coarse-grid correction factor (multigrid.hpp:1898-1925): MinEnergy
// omega = (def . cor) / (tmp . cor), MinDefect omega = (def . tmp) / (tmp . tmp), tmp = A cor;
// both sums in one pass, deterministic (partials per CTA, summed in order by the last CTA)
template<typename T>
__global__ void __launch_bounds__(256) k_cgc_omega(const T* __restrict__ def, const T* __restrict__ cor,
                                                   const T* __restrict__ tmp, uint32_t n, int min_defect,
                                                   double* ws, unsigned* counter, double* omega) {
  __shared__ double sh[8];
  __shared__ bool am_last;
  double a = 0.0, b = 0.0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double t = double(tmp[i]);
    if (min_defect) { a += double(def[i]) * t; b += t * t; }
    else { const double c = double(cor[i]); a += double(def[i]) * c; b += t * c; }
  }
  const double ba = block_sum<256>(a, sh);
  __syncthreads();
  const double bb = block_sum<256>(b, sh);
  if (threadIdx.x == 0) {
    ws[blockIdx.x] = ba;
    ws[gridDim.x + blockIdx.x] = bb;
    __threadfence();
    am_last = atomicAdd(counter, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!am_last) return;
  __threadfence();
  double va = 0.0, vb = 0.0;
  for (unsigned i = threadIdx.x; i < gridDim.x; i += 256) { va += __ldcg(ws + i); vb += __ldcg(ws + gridDim.x + i); }
  va = block_sum<256>(va, sh);
  __syncthreads();
  vb = block_sum<256>(vb, sh);
  if (threadIdx.x == 0) {
    *omega = va / vb;
    *counter = 0u;
  }
}

// sol += omega * cor (the correction is already filtered)
template<typename T>
__global__ void k_cgc_update(T* sol, const T* __restrict__ cor, const double* omega, uint32_t n) {
  const T w = T(*omega);
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    sol[i] = w * cor[i] + sol[i];
}

// Richardson outer: x = omega * z + x
template<typename ZT>
__global__ void k_rich_update(double* x, const ZT* __restrict__ z, double omega, uint32_t n) {
  if (fabs(omega) < eps_of<double>()) return;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    x[i] = omega * double(z[i]) + x[i];
}

template<typename T>
__global__ void k_fill(T* x, T v, uint32_t n) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) x[i] = v;
}

__global__ void k_invdiag(double* invd64, float* invd32, const double* __restrict__ diag, double omega, uint32_t n) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double v = omega / diag[i];
    if (invd64) invd64[i] = v;
    if (invd32) invd32[i] = float(omega) / float(diag[i]);
  }
}

template<typename D, typename S>
__global__ void k_cvt(D* d, const S* __restrict__ s, uint64_t n) {
  for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x) d[i] = D(s[i]);
}

__global__ void k_absmax(const double* __restrict__ v, uint64_t n, unsigned long long* out) {
  double m = 0.0;
  for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x)
    m = fmax(m, fabs(v[i]));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, __double_as_longlong(m));  // non-negative doubles order as integers
}

// the SELL form's FP16 values: slot pairs of every chunk interleaved (k_sell's FP16 layout), one
// warp per chunk
__global__ void k_quant16_sell(__half* d, const double* __restrict__ s, double inv, const uint32_t* __restrict__ cs,
                               const uint32_t* __restrict__ cl, uint32_t nchunks) {
  const uint32_t lane = threadIdx.x & 31;
  for (uint32_t c = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; c < nchunks; c += (gridDim.x * blockDim.x) >> 5) {
    const uint32_t beg = cs[c], len = cl[c], even = len & ~1u;
    for (uint32_t j = 0; j < len; ++j) {
      const uint32_t src = beg + j * 32u + lane;
      const uint32_t dst = j < even ? beg + (j >> 1) * 64u + 2u * lane + (j & 1u) : src;
      d[dst] = __double2half(s[src] * inv);
    }
  }
}

unsigned ew_grid(uint64_t n) {
  unsigned g = grid_for(n, 256);
  return g > 8u * kSMs ? 8u * kSMs : g;
}

// ------------------------------------------------------------------ V-cycle
template<typename T> struct Prec;
template<> struct Prec<double> {
  static double* rhs(Level& l) { return l.rhs64; }
  static double* x(Level& l) { return l.x64; }
  static double* y(Level& l) { return l.y64; }
  static double* def(Level& l) { return l.def64; }
  static double* invd(Level& l) { return l.invd64; }
  static double* cor(Level& l) { return l.cor64; }
  static double* tmp(Level& l) { return l.tmp64; }
};
template<> struct Prec<float> {
  static float* rhs(Level& l) { return l.rhs32; }
  static float* x(Level& l) { return l.x32; }
  static float* y(Level& l) { return l.y32; }
  static float* def(Level& l) { return l.def32; }
  static float* invd(Level& l) { return l.invd32; }
  static float* cor(Level& l) { return l.cor32; }
  static float* tmp(Level& l) { return l.tmp32; }
};

// dispatch a SELL launch on the value storage of the configured precision
static bool use_stencil(const fb_mg* m, const Level& L) {
  return m->cfg.format != FB_FORMAT_SELL && L.St.S > 0;
}
static bool use_matfree(const fb_mg* m, const Level& L) {
  return m->cfg.format == FB_FORMAT_MATFREE && L.mf;
}
// the structured formats replace the CSR transfer matrices by the matrix-free Q1 transfers
static bool use_q1_transfer(const fb_mg* m, const Level& L) {
  return m->cfg.format != FB_FORMAT_SELL && L.q1_transfer;
}

// self-check record of the matrix-free kernels (FB_CHECK=1): report and clear it
static int check_self_checks(fb_mg* m) {
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(m->stream, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) return FB_OK;
  unsigned long long h = 0;
  FB_CUDA(cudaMemcpyAsync(&h, m->dbg_err, sizeof(h), cudaMemcpyDeviceToHost, m->stream));
  FB_CUDA(cudaStreamSynchronize(m->stream));
  if (!h) return FB_OK;
  FB_CUDA(cudaMemsetAsync(m->dbg_err, 0, sizeof(h), m->stream));
  const unsigned kind = unsigned(h >> 62);
  std::fprintf(stderr, "feat3_b200: k_mf_q1 self-check: %s (row %llu, slot %llu)\n",
               kind == 1 ? "x index out of range" : (kind == 2 ? "cell index out of range" : "geometry mismatch"),
               (h >> 8) & 0xffffffffull, h & 0xffull);
  return FB_ERR_CUDA;
}

// line-tiled staged launch (3D levels with at least 16 interior points per line)
template<typename T, typename Epi, int TY, int NST, int MINB, int CM1, typename XT = T>
static int launch_mf_tiled_ty(fb_mg* m, const Level& L, const MfView<T, 3>& v, const XT* x, const Epi& epi,
                              double* red_out) {
  using SE = Staged<Epi>;
  constexpr int NS = SE::kStreams;
  const uint32_t M1 = L.M1, N = M1 - 1, W = M1 - 2;
  auto r16 = [](uint64_t b) { return uint32_t((b + 15) & ~uint64_t(15)); };
  // a structured level's filter is its lattice boundary, which no tile row touches
  const uint32_t* mask = (L.mask_boundary && SE::mask(epi) == L.mask) ? nullptr : SE::mask(epi);
  MfTile G;
  G.M1 = M1; G.N = N;
  G.G = std::max<uint32_t>(1, 256 / W);
  G.Lt = G.G * TY;
  G.tpp = (W + G.Lt - 1) / G.Lt;
  G.ntiles = W * G.tpp;
  G.cap_x = r16(uint64_t(G.Lt + 2) * M1 * sizeof(XT)) + 32;
  G.cap_k = v.k ? r16(uint64_t(G.Lt + 1) * N * sizeof(T)) + 32 : 0;
  G.cap_s = NS ? r16(uint64_t(G.Lt) * M1 * sizeof(T)) + 32 : 0;
  G.cap_m = mask ? r16((uint64_t(G.Lt) * M1 / 32 + 2) * 4) + 32 : 0;
  G.stage_bytes = (3 * G.cap_x + 2 * G.cap_k + NS * G.cap_s + G.cap_m + 127) & ~127u;
  G.nbl_items = (4 * M1 - 4) * ((M1 + 31) / 32);
  G.nedge_items = (W * W + 15) / 16;
  G.direct_masked = (L.mask_boundary && L.mask && SE::mask(epi) == L.mask) ? 1u : 0u;
  G.inject = m->inject;
  const size_t dyn = size_t(NST) * G.stage_bytes;
  auto fn = k_mf_q1_tiled<T, Epi, NST, MINB, TY, CM1, XT>;
  static size_t attr = 0;  // per instantiation: largest dynamic shared memory requested so far
  if (dyn > attr) {
    FB_CUDA(cudaFuncSetAttribute((const void*)fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(dyn)));
    attr = dyn;
  }
  int bps = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, (const void*)fn, 288, dyn) != cudaSuccess || bps < 1) {
    cudaGetLastError();
    bps = 1;
  }
  const uint32_t grid = std::max<uint32_t>(1, std::min<uint32_t>(G.ntiles, uint32_t(bps) * kSMs));
  G.dz = grid / G.tpp;
  G.dyt = grid % G.tpp;
  const T* s0 = NS > 0 ? static_cast<const T*>(SE::stream(epi, 0)) : nullptr;
  const T* s1 = NS > 1 ? static_cast<const T*>(SE::stream(epi, 1)) : nullptr;
  FB_CUDA(launch_pdl(m->stream, fn, dim3(grid), dim3(288), dyn, v, G, x, epi, s0, s1, mask, m->ws, m->counter, red_out,
                     m->kerr));
  m->launches++;
  FB_CHECK_LAUNCH();
  return FB_OK;
}

// streaming launch (levels of 257^3 and 129^3 points, filter = the lattice boundary): NST stages of
// TY lines, NCW consumer warps per CTA (8: MINB CTAs per SM; 12 or 16: one), CPT rows per thread;
// one contiguous range of slab-lines per CTA
template<typename T, typename Epi, int TY, int NST, int CM1, typename XT = T, int NCW = 8, int MINB = 2, int CPT = 1>
static int launch_mf_stream(fb_mg* m, const Level& L, const MfView<T, 3>& v, const XT* x, const Epi& epi,
                            double* red_out) {
  using SE = Staged<Epi>;
  constexpr int NS = SE::kStreams;
  constexpr uint32_t M1 = CM1, N = M1 - 1, W = M1 - 2;
  constexpr int NT = 32 * (NCW + 1);
  constexpr uint32_t PW = (W + CPT - 1) / CPT;  // consumer threads per line
  auto r16 = [](uint64_t b) { return uint32_t((b + 15) & ~uint64_t(15)); };
  MfStream G{};
  G.G = std::max<uint32_t>(1, uint32_t(32 * NCW) / PW);
  G.nslab = (W + G.G - 1) / G.G;
  G.units = uint64_t(G.nslab) * W;
  G.cap_x = r16(uint64_t(TY) * M1 * sizeof(XT)) + 32;
  G.cap_k = v.k ? r16(uint64_t(TY) * N * sizeof(T)) + 32 : 0;
  G.cap_s = NS ? r16(uint64_t(TY) * M1 * sizeof(T)) + 32 : 0;
  G.stage_bytes = ((G.G + 2) * G.cap_x + (G.G + 1) * G.cap_k + NS * G.G * G.cap_s + 127) & ~127u;
  G.nbl_items = (4 * M1 - 4) * ((M1 + 31) / 32);
  G.nedge_items = (W * W + 15) / 16;
  G.direct_masked = (L.mask && SE::mask(epi) == L.mask) ? 1u : 0u;
  G.inject = m->inject;
  const size_t dyn = size_t(NST) * G.stage_bytes;
  static_assert(NCW == 8 || NCW == 12 || NCW == 16, "8, 12 or 16 consumer warps");
  void (*fn)(MfView<T, 3>, MfStream, const XT*, Epi, const T*, const T*, double*, unsigned*, double*, unsigned*);
  if constexpr (NCW == 8) fn = k_mf_q1_stream<T, Epi, NST, MINB, TY, CM1, XT, CPT>;
  else if constexpr (NCW == 12) fn = k_mf_q1_stream12<T, Epi, NST, TY, CM1, XT, CPT>;
  else fn = k_mf_q1_stream16<T, Epi, NST, TY, CM1, XT, CPT>;
  static size_t attr = 0;  // per instantiation: largest dynamic shared memory requested so far
  if (dyn > attr) {
    FB_CUDA(cudaFuncSetAttribute((const void*)fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(dyn)));
    attr = dyn;
  }
  int bps = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, (const void*)fn, NT, dyn) != cudaSuccess || bps < 1) {
    cudaGetLastError();
    bps = 1;
  }
  const uint32_t grid = uint32_t(std::min<uint64_t>(G.units, uint64_t(bps) * kSMs));
  const T* s0 = NS > 0 ? static_cast<const T*>(SE::stream(epi, 0)) : nullptr;
  const T* s1 = NS > 1 ? static_cast<const T*>(SE::stream(epi, 1)) : nullptr;
  FB_CUDA(launch_pdl(m->stream, fn, dim3(grid), dim3(NT), dyn, v, G, x, epi, s0, s1, m->ws, m->counter, red_out,
                     m->kerr));
  m->launches++;
  FB_CHECK_LAUNCH();
  return FB_OK;
}

// the streaming kernel takes the FP32 forms on the levels of 257^3 and 129^3 points whose filter is
// the lattice boundary (Jacobi step 74.7 against 82.5 us, defect 67.7 against 71.8 us per level-8
// launch, same box). PCG's FP64 q = A p from the FP32 direction stays on the tiled kernel: its
// streaming form spills at the 96 registers of two CTAs per SM (111.4 against 96.4 us).
template<typename T, typename Epi, typename XT>
static bool stream_ok(const fb_mg* m, const Level& L, const Epi& epi) {
  const bool form = std::is_same<T, float>::value && std::is_same<XT, float>::value;
  const uint32_t* mask = Staged<Epi>::mask(epi);
  return form && (L.M1 == 257 || L.M1 == 129) && L.mask_boundary && (mask == nullptr || mask == L.mask) &&
         !(m->cfg.flags & FB_FLAG_NO_STREAM);
}

// lines per thread and CTAs per SM (measured on the 257^3 solve): FP32 6 lines, 2 CTAs (96
// registers, no spills; 4 lines at 3 CTAs spilled and ran 2.5 % slower); FP64 2 lines, 2 CTAs
// (4 % faster than 3 lines), except PCG's q = A p with no streamed inputs: 3 lines (123 us per
// level-8 launch against 149 us with 2 lines and 222 us with 1); the same from the FP32-stored
// direction, whose stages are smaller: 6 lines (101 us against 120 us with 3, 110 us with 4).
// Levels 8 and 7 of the 3D hierarchy get the lattice size as a compile-time constant (3.5 %
// faster solve than the run-time size). FP32 on the smaller levels (65^3 and below): 2 lines
// per thread (17.33 vs 17.51 ms with 6; at 33^3 a plane of 31 lines is otherwise a single tile).
template<typename T, typename Epi, typename XT = T>
static int launch_mf_tiled(fb_mg* m, const Level& L, const MfView<T, 3>& v, const XT* x, const Epi& epi,
                           double* red_out) {
  // FP64 PCG-q from an FP64 direction: 3 lines; from the FP32 direction (smaller stages): 6
  constexpr int TY = sizeof(T) == 4 ? 6
                     : std::is_same<Epi, EpiPcgQ<double, float>>::value ? 6
                     : std::is_same<Epi, EpiPcgQ<double>>::value ? 3 : 2;
  // at 257^3: the FP32 defect streams one vector, 8 lines fit one CTA per SM and ran faster
  // (65.6 us against 71.3 us with 6 lines at two CTAs); the FP32 Jacobi step with the diagonal
  // from the coefficients streams one vector too, 7 lines still fit two CTAs per SM (solve
  // 15.05 ms against 15.17 ms with 6 lines, same box)
  constexpr int TY8 = std::is_same<Epi, EpiDefect<float, false, false>>::value ? 8
                      : (std::is_same<Epi, EpiJacobiK<float, false, false>>::value ||
                         std::is_same<Epi, EpiJacobiK<float, true, false>>::value ||
                         std::is_same<Epi, EpiJacobiK<float, false, true>>::value) ? 7 : TY;
  if constexpr (std::is_same<T, float>::value && std::is_same<XT, float>::value) {
    if (stream_ok<T, Epi, XT>(m, L, epi)) {
      // 257^3, at most one streamed vector: one CTA of 12 consumer warps per SM, two adjacent rows
      // per thread (slabs of three planes), 3 stages of 6 lines: Jacobi step 64.0 us, defect 60.8
      // us per launch, solve 14.57 ms (with the boundary rows left out of both forms, 61.6 against
      // 64.5 us per Jacobi step with one row per thread and 16 warps). Two streamed vectors: one
      // CTA of 16 warps, one row per thread (slabs of two planes share their x planes), 3 stages
      // (one CTA of 16 warps with 4 stages ran the solve in 15.21 against 15.40 ms with two CTAs
      // of 8 warps, same box). 129^3: two CTAs of 8 warps, 3 stages (14.5 against 16.2 us per
      // launch)
      if constexpr (Staged<Epi>::kStreams <= 1) {
        if (L.M1 == 257) return launch_mf_stream<T, Epi, 6, 3, 257, XT, 12, 1, 2>(m, L, v, x, epi, red_out);
      }
      constexpr int NSTW = Staged<Epi>::kStreams > 1 ? 3 : 4;
      if (L.M1 == 257) return launch_mf_stream<T, Epi, 6, NSTW, 257, XT, 16, 1>(m, L, v, x, epi, red_out);
      return launch_mf_stream<T, Epi, 6, 3, 129, XT>(m, L, v, x, epi, red_out);
    }
  }
  if (L.M1 == 257) return launch_mf_tiled_ty<T, Epi, TY8, 2, 2, 257, XT>(m, L, v, x, epi, red_out);
  if (L.M1 == 129) return launch_mf_tiled_ty<T, Epi, TY, 2, 2, 129, XT>(m, L, v, x, epi, red_out);
  // the smaller levels have few lines per plane: short tiles spread them over more CTAs
  constexpr int TYS = sizeof(T) == 4 ? 2 : TY;
  return launch_mf_tiled_ty<T, Epi, TYS, 2, 2, 0, XT>(m, L, v, x, epi, red_out);
}

// the FP32 Jacobi step whose tiled form takes its inverse diagonal from the cell coefficients
template<typename Epi> struct JacobiK { using type = void; };
template<bool RED, bool DOT> struct JacobiK<EpiJacobi<float, RED, DOT>> { using type = EpiJacobiK<float, RED, DOT>; };

template<typename T, typename Epi, int DIM>
static int launch_mf_D(fb_mg* m, const Level& L, const T* x, const Epi& epi, double* red_out) {
  MfView<T, DIM> v;
  v.rows = L.n; v.nchunks = (L.n + 31) / 32; v.M1 = L.M1; v.ne = L.ne;
  v.err = check_enabled() ? m->dbg_err : nullptr;
  if constexpr (std::is_same<T, double>::value) {
    v.k = L.k;
    for (int r = 0; r < (1 << DIM); ++r) v.kr[r] = L.kr64[r];
  } else {
    v.k = L.k ? L.k32 : nullptr;
    for (int r = 0; r < (1 << DIM); ++r) v.kr[r] = L.kr32[r];
  }
  for (int j = 0; j < (DIM == 3 ? 27 : 9); ++j) v.off[j] = L.St.off[j];
  if constexpr (DIM == 3 && Staged<Epi>::kOk) {
    if (L.M1 >= 18 && L.n < (1u << 31) && Staged<Epi>::input_is_x(epi, x) && !v.err && m->mf_faces0 &&
        !(m->cfg.flags & FB_FLAG_NO_TILED)) {
      using EK = typename JacobiK<Epi>::type;
      if constexpr (!std::is_void<EK>::value) {
        // the level's stored inverse diagonal is omega_jac / (kr[0] * sum of the row's 8 k):
        // formed in the kernel, one streamed vector less (solve 15.17 ms against 15.23 ms with
        // the stored one at 6 lines, same box; the FP32 V-cycle is the preconditioner, and
        // __fdividef's few-ulp quotient leaves the iteration count unchanged)
        if (epi.invd == L.invd32) {
          EK ek;
          static_cast<Epi&>(ek) = epi;
          ek.wd = float(m->cfg.omega_jac) / v.kr[0];
          return launch_mf_tiled<T, EK>(m, L, v, x, ek, red_out);
        }
      }
      return launch_mf_tiled<T, Epi>(m, L, v, x, epi, red_out);
    }
  }
  auto fn = k_mf_q1<T, Epi, DIM>;
  if (debug_enabled())
    debug_check_ptrs("k_mf_q1", {(const void*)v.k, (const void*)x, (const void*)m->ws, (const void*)m->counter,
                                 (const void*)red_out});
  FB_CUDA(launch_pdl(m->stream, fn, dim3(occupancy_grid((const void*)fn, v.nchunks)), dim3(256), 0, v, x, epi, m->ws,
                     m->counter, red_out));
  m->launches++;
  FB_CHECK_LAUNCH();
  if (v.err && debug_enabled()) FB_TRY(check_self_checks(m));
  return FB_OK;
}

// The mixed matrix-free form keeps PCG's search direction in FP32 (half the bytes of p in the
// direction update and in q = A p; the product itself in FP64): 3D levels the tiled kernel takes.
static bool pcg_p32(const fb_mg* m) {
  if (m->cfg.outer != FB_OUTER_PCG || m->cfg.precision == FB_PREC_F64 || m->dim != 3) return false;
  const Level& L = m->L[0];
  return use_matfree(m, L) && L.M1 >= 18 && L.n < (1u << 31) && m->mf_faces0 && !check_enabled() &&
         !(m->cfg.flags & FB_FLAG_NO_TILED);
}

// q = filter_def(A p) and q . p with p stored in FP32, A(k) in FP64 (finest level)
static int pcgq_p32(fb_mg* m, double* red, const float* p) {
  const Level& L = m->L[0];
  MfView<double, 3> v;
  v.rows = L.n; v.nchunks = (L.n + 31) / 32; v.M1 = L.M1; v.ne = L.ne;
  v.err = nullptr;
  v.k = L.k;
  for (int r = 0; r < 8; ++r) v.kr[r] = L.kr64[r];
  for (int j = 0; j < 27; ++j) v.off[j] = L.St.off[j];
  EpiPcgQ<double, float> eq{m->q, p, L.mask};
  return launch_mf_tiled<double, EpiPcgQ<double, float>, float>(m, L, v, p, eq, red);
}

// level operator A x with an epilogue, on the storage the configuration selects
template<typename T, typename Epi>
static int spmv_L(fb_mg* m, const Level& L, const T* x, const Epi& epi, double* red) {
  if (use_matfree(m, L)) {
    if (m->dim == 3) return launch_mf_D<T, Epi, 3>(m, L, x, epi, red);
    return launch_mf_D<T, Epi, 2>(m, L, x, epi, red);
  }
  const bool st = use_stencil(m, L);
  if constexpr (std::is_same<T, double>::value) {
    if (st) return launch_stencil<double, double, double, Epi>(m, L, FB_PREC_F64, x, epi, red);
    return launch_sell<double, double, double, Epi>(m, L.A, FB_PREC_F64, x, epi, red);
  } else {
    if (m->cfg.precision == FB_PREC_F16) {
      if (st) return launch_stencil<__half, float, float, Epi>(m, L, FB_PREC_F16, x, epi, red);
      return launch_sell<__half, float, float, Epi>(m, L.A, FB_PREC_F16, x, epi, red);
    }
    if (st) return launch_stencil<float, float, float, Epi>(m, L, FB_PREC_F32, x, epi, red);
    return launch_sell<float, float, float, Epi>(m, L.A, FB_PREC_F32, x, epi, red);
  }
}

// bulk-staged 3D restriction onto a coarse level whose filter is its lattice boundary: tiles of
// TYC coarse lines per thread group, 2-deep ring, as many CTAs as fit (2 per SM at 129^3)
template<typename T, int TYC, int NST = 2>
static int launch_rest_staged(fb_mg* m, const Level& L, const T* xf, const EpiRestrict<T>& epi, double* red) {
  const uint32_t Mc1 = L.tr.Mc1, Mf1 = L.tr.Mf1, Wc = Mc1 - 2;
  MfTile G{};
  G.M1 = Mc1; G.N = Mc1 - 1;
  G.G = std::max<uint32_t>(1, 256 / Wc);
  G.Lt = G.G * TYC;
  G.tpp = (Wc + G.Lt - 1) / G.Lt;
  G.ntiles = Wc * G.tpp;
  G.cap_x = uint32_t(((uint64_t(2 * G.Lt + 1) * Mf1 * sizeof(T) + 15) & ~uint64_t(15)) + 32);
  G.stage_bytes = (3 * G.cap_x + 127) & ~127u;
  G.nbl_items = (4 * Mc1 - 4) * ((Mc1 + 31) / 32);
  G.nedge_items = (Wc * Wc + 15) / 16;
  G.direct_masked = 1;
  const size_t dyn = size_t(NST) * G.stage_bytes;
  auto fn = k_rest_q1_staged<T, NST, TYC>;
  static size_t attr = 0;  // per instantiation: largest dynamic shared memory requested so far
  if (dyn > attr) {
    FB_CUDA(cudaFuncSetAttribute((const void*)fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(dyn)));
    attr = dyn;
  }
  int bps = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, (const void*)fn, 288, dyn) != cudaSuccess || bps < 1) {
    cudaGetLastError();
    bps = 1;
  }
  const uint32_t grid = std::max<uint32_t>(1, std::min<uint32_t>(G.ntiles, uint32_t(bps) * kSMs));
  G.dz = grid / G.tpp;
  G.dyt = grid % G.tpp;
  FB_CUDA(launch_pdl(m->stream, fn, dim3(grid), dim3(288), dyn, G, Mf1, xf, epi, m->ws, m->counter, red, m->kerr));
  m->launches++;
  FB_CHECK_LAUNCH();
  return FB_OK;
}

// restriction from level l onto level l+1 (R d), epilogue on the coarse rows
template<typename T, typename Epi>
static int rest_T(fb_mg* m, int l, const T* xf, const Epi& epi, double* red) {
  const Level& L = m->L[l];
  if (use_q1_transfer(m, L)) {
    if constexpr (std::is_same<Epi, EpiRestrict<T>>::value) {
      if (L.tr.dim == 3) {
        constexpr int CZ = sizeof(T) == 4 ? 4 : 2;  // static shared tile below 48 KB
        // coarse level l+1: its filter is the lattice boundary when structured
        const int bmask = m->L[l + 1].mask_boundary && epi.mask == m->L[l + 1].mask;
        // staged by bulk copies (257^3 solve, same box: 15.97 ms with k_rest_q1_tile on every
        // level, 15.73 ms staged onto 65^3 and up, 15.62 ms staged onto 17^3 and up); coarse
        // lines per thread: FP32 onto 129^3 and up 4 (17 fine lines of a stage), 2 onto 65^3
        // and up, 1 below (more tiles for the CTAs)
        if (bmask && L.tr.Mc1 >= 17 && L.tr.nf < (1u << 31)) {
          if (sizeof(T) == 4 && L.tr.Mc1 >= 129) return launch_rest_staged<T, 4>(m, L, xf, epi, red);
          if (L.tr.Mc1 >= 65) return launch_rest_staged<T, 2>(m, L, xf, epi, red);
          return launch_rest_staged<T, 1>(m, L, xf, epi, red);
        }
        const uint32_t E = L.tr.Mc1 - (bmask ? 1 : 0);  // indices the grid must cover
        // below 129^3 coarse points, 2 coarse planes per block spread the few blocks better
        // (8.6 vs 12.2 us onto 17^3; 47.8 vs 50.4 us onto 129^3 stays with 4)
        if (CZ == 4 && L.tr.Mc1 < 129) {
          const dim3 g2((E + 31) / 32, (E + 7) / 8, (E + 1) / 2);
          FB_CUDA(launch_pdl(m->stream, k_rest_q1_tile<T, 2>, g2, dim3(256), 0, L.tr, xf, epi, m->ws, m->counter, red,
                             bmask));
        } else {
          const dim3 grid((E + 31) / 32, (E + 7) / 8, (E + CZ - 1) / CZ);
          FB_CUDA(launch_pdl(m->stream, k_rest_q1_tile<T, CZ>, grid, dim3(256), 0, L.tr, xf, epi, m->ws, m->counter,
                             red, bmask));
        }
        m->launches++;
        FB_CHECK_LAUNCH();
        return FB_OK;
      }
    }
    const dim3 grid((L.tr.Mc1 + 31) / 32, (L.tr.Mc1 + 7) / 8, L.tr.dim == 3 ? L.tr.Mc1 : 1);
    k_rest_q1<T, Epi><<<grid, dim3(32, 8), 0, m->stream>>>(L.tr, xf, epi, m->ws, m->counter, red);
    m->launches++;
    FB_CHECK_LAUNCH();
    return FB_OK;
  }
  if constexpr (std::is_same<T, double>::value) return launch_csr<double, double, double, Epi>(m, L.R, false, xf, epi, red);
  else return launch_csr<float, float, float, Epi>(m, L.R, true, xf, epi, red);
}

// prolongation from level l+1 onto level l (P x_c), epilogue on the fine rows
template<typename T, typename Epi>
static int prol_T(fb_mg* m, int l, const T* xc, const Epi& epi) {
  const Level& L = m->L[l];
  if (use_q1_transfer(m, L)) {
    if constexpr (std::is_same<Epi, EpiProlong<T>>::value) {
      if (L.tr.dim == 3) {
        constexpr int FZ = 8;  // 8 fine planes per thread: measured fastest of 4 / 8 / 16
        const int bmask = L.mask_boundary && epi.mask == L.mask;
        // filtered rows take no correction: with the boundary filter the grid skips the last
        // plane, line and column (2^l + 1 points per side) instead of spending a block on each
        const uint32_t E = L.tr.Mf1 - (bmask ? 1 : 0);
        const dim3 grid((E + 31) / 32, (E + 7) / 8, (E + FZ - 1) / FZ);
        FB_CUDA(launch_pdl(m->stream, k_prol_q1_tile<T, FZ>, grid, dim3(256), 0, L.tr, xc, epi.sol, epi.mask, bmask));
        m->launches++;
        FB_CHECK_LAUNCH();
        return FB_OK;
      }
    }
    const dim3 grid((L.tr.Mf1 + 31) / 32, (L.tr.Mf1 + 7) / 8, L.tr.dim == 3 ? L.tr.Mf1 : 1);
    k_prol_q1<T, Epi><<<grid, dim3(32, 8), 0, m->stream>>>(L.tr, xc, epi);
    m->launches++;
    FB_CHECK_LAUNCH();
    return FB_OK;
  }
  if constexpr (std::is_same<T, double>::value) return launch_csr<double, double, double, Epi>(m, L.P, false, xc, epi, nullptr);
  else return launch_csr<float, float, float, Epi>(m, L.P, true, xc, epi, nullptr);
}

// pre-smoothing from zero with rhs b on level l (Richardson(Jacobi), nu steps); `cur` holds
// s1 on entry unless `need_s1`; returns the buffer with the smoothed iterate
template<typename T>
static int presmooth(fb_mg* m, int l, const T* b, const double* bnorm, bool need_s1, T** result) {
  Level& L = m->L[l];
  const T omega = T(m->cfg.omega_rich);
  T* cur = Prec<T>::x(L);
  T* oth = Prec<T>::y(L);
  if (need_s1) {
    k_jacobi0<T><<<ew_grid(L.n), 256, 0, m->stream>>>(cur, b, Prec<T>::invd(L), L.mask, bnorm, omega, L.n);
    m->launches++;
    FB_CHECK_LAUNCH();
  }
  for (int it = 1; it < m->cfg.nu; ++it) {
    EpiJacobi<T, false> e{cur, b, Prec<T>::invd(L), oth, nullptr, L.mask, bnorm, omega};
    FB_TRY(spmv_L<T>(m, L, cur, e, nullptr));
    std::swap(cur, oth);
  }
  *result = cur;
  return FB_OK;
}

// ------------------------------------------------------------------ fused coarse cycle
// levels up to this size go to the one-cluster kernel: 3D level 4 (4,913 rows) and below. The
// 3D level 5 (35,937 rows) runs faster as separate full-GPU launches (measured: 19.8 vs 20.3 ms
// for the 257^3 mixed solve), since the cluster's 16 SMs are latency-bound on it.
constexpr uint32_t kCoarseRows = 5000;
template<typename T> constexpr int coarse_threads() { return 512; }

template<typename T, int DIM>
static int coarse_cluster_size(fb_mg* m) {
  // largest cluster (16 non-portable, else 8) that the device can schedule for the kernel
  static int cs = -1;
  if (cs >= 0) return cs;
  cs = 0;
  auto fn = k_coarse_cycle<T, DIM, coarse_threads<T>()>;
  (void)m;
  for (int want : {16, 8}) {
    if (want > 8 && cudaFuncSetAttribute((const void*)fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) {
      cudaGetLastError();
      continue;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(want);
    cfg.blockDim = dim3(coarse_threads<T>());
    cudaLaunchAttribute at;
    at.id = cudaLaunchAttributeClusterDimension;
    at.val.clusterDim.x = want; at.val.clusterDim.y = 1; at.val.clusterDim.z = 1;
    cfg.attrs = &at;
    cfg.numAttrs = 1;
    int nc = 0;
    if (cudaOccupancyMaxActiveClusters(&nc, (const void*)fn, &cfg) == cudaSuccess && nc > 0) { cs = want; break; }
    cudaGetLastError();
  }
  return cs;
}

// first level of the fused coarse cycle, or nl when the coarse end runs level by level
template<typename T>
static int coarse_start(fb_mg* m) {
  const int nl = (int)m->L.size();
  if (m->cfg.format != FB_FORMAT_MATFREE || m->cfg.coarse == FB_COARSE_PCG || (m->cfg.flags & FB_FLAG_NO_COARSE_FUSION))
    return nl;
  int lc = nl;
  for (int l = nl - 1; l >= 1; --l) {
    if (!m->L[l].mf || m->L[l].n > kCoarseRows) break;
    lc = l;
  }
  if (nl - lc < 2 || nl - lc > kCoarseMax) return nl;
  const int cs = m->dim == 3 ? coarse_cluster_size<T, 3>(m) : coarse_cluster_size<T, 2>(m);
  return cs > 0 ? lc : nl;
}

template<typename T>
static int launch_coarse(fb_mg* m, int lc, T** sol_lc) {
  const int nl = (int)m->L.size();
  CoarseArgs<T> A;
  A.nlv = nl - lc;
  A.nu = m->cfg.nu;
  A.coarse = m->cfg.coarse;
  A.omega = T(m->cfg.omega_rich);
  if constexpr (std::is_same<T, double>::value) A.cinv = m->cinv64; else A.cinv = m->cinv32;
  A.s1_coarsest = m->cfg.coarse == FB_COARSE_SMOOTHER ? 1 : 0;
  for (int i = 0; i < A.nlv; ++i) {
    Level& L = m->L[lc + i];
    CLevel<T>& c = A.L[i];
    c.n = L.n; c.M1 = L.M1;
    if constexpr (std::is_same<T, double>::value) {
      c.k = L.k;
      for (int r = 0; r < 8; ++r) c.kr[r] = L.kr64[r];
    } else {
      c.k = L.k ? L.k32 : nullptr;
      for (int r = 0; r < 8; ++r) c.kr[r] = L.kr32[r];
    }
    c.mask = L.mask; c.invd = Prec<T>::invd(L);
    c.rhs = Prec<T>::rhs(L); c.x = Prec<T>::x(L); c.y = Prec<T>::y(L); c.def = Prec<T>::def(L);
    c.bn = &m->sc->lvl[2 * (lc + i)];
    c.dn = &m->sc->lvl[2 * (lc + i) + 1];
  }
  const int cs = m->dim == 3 ? coarse_cluster_size<T, 3>(m) : coarse_cluster_size<T, 2>(m);
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(cs);
  cfg.blockDim = dim3(coarse_threads<T>());
  cfg.stream = m->stream;
  cudaLaunchAttribute at[2];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = cs; at[0].val.clusterDim.y = 1; at[0].val.clusterDim.z = 1;
  at[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[1].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = pdl_enabled() ? 2 : 1;
  if (m->dim == 3) FB_CUDA(cudaLaunchKernelEx(&cfg, k_coarse_cycle<T, 3, coarse_threads<T>()>, A));
  else FB_CUDA(cudaLaunchKernelEx(&cfg, k_coarse_cycle<T, 2, coarse_threads<T>()>, A));
  m->launches++;
  FB_CHECK_LAUNCH();
  // the kernel's pointer walk: nu - 1 swaps in the pre-smoothing of level lc, nu in its post-smoothing
  Level& L = m->L[lc];
  T* cur = Prec<T>::x(L);
  for (int it = 1; it < m->cfg.nu; ++it) cur = (cur == Prec<T>::x(L)) ? Prec<T>::y(L) : Prec<T>::x(L);
  for (int it = 0; it < m->cfg.nu; ++it) cur = (cur == Prec<T>::x(L)) ? Prec<T>::y(L) : Prec<T>::x(L);
  *sol_lc = cur;
  return FB_OK;
}

template<typename T>
static int vcycle(fb_mg* m, const T* rhs_top, const double* rhs_top_sumsq, T** out_top) {
  const int nl = (int)m->L.size();
  const int nu = m->cfg.nu;
  const T omega = T(m->cfg.omega_rich);
  std::vector<T*> sol(nl, nullptr);
  const int lc = coarse_start<T>(m);
  // ---- descent (multigrid.hpp:1711-1832)
  for (int l = 0; l + 1 < nl && l < lc; ++l) {
    Level& L = m->L[l];
    Level& C = m->L[l + 1];
    const T* b = (l == 0) ? rhs_top : Prec<T>::rhs(L);
    const double* bn = (l == 0) ? rhs_top_sumsq : &m->sc->lvl[2 * l];
    const bool need_s1 = (l == 0) ? !m->top_s1 : nu < 2;
    FB_TRY(presmooth<T>(m, l, b, bn, need_s1, &sol[l]));
    EpiDefect<T, false, false> ed{Prec<T>::def(L), b, L.mask, nullptr};
    FB_TRY(spmv_L<T>(m, L, sol[l], ed, nullptr));
    const bool coarsest_next = (l + 2 == nl);
    T* s1 = nullptr;
    if (nu >= 2 && (!coarsest_next || m->cfg.coarse == FB_COARSE_SMOOTHER)) s1 = Prec<T>::x(C);
    EpiRestrict<T> er{Prec<T>::rhs(C), s1, Prec<T>::invd(C), C.mask, omega};
    FB_TRY(rest_T<T>(m, l, Prec<T>::def(L), er, &m->sc->lvl[2 * (l + 1)]));
  }
  // ---- coarse grid (multigrid.hpp:1524-1587)
  if (lc < nl) {
    FB_TRY(launch_coarse<T>(m, lc, &sol[lc]));
  } else {
    const int l = nl - 1;
    Level& L = m->L[l];
    const T* b = (l == 0) ? rhs_top : Prec<T>::rhs(L);
    const double* bn = (l == 0) ? rhs_top_sumsq : &m->sc->lvl[2 * l];
    switch (m->cfg.coarse) {
      case FB_COARSE_DIRECT: {
        const T* cinv;
        if constexpr (std::is_same<T, double>::value) cinv = m->cinv64; else cinv = m->cinv32;
        k_dense_solve<T><<<grid_for(uint64_t(L.n) * 32, 256), 256, 0, m->stream>>>(Prec<T>::x(L), cinv, b, L.n);
        m->launches++;
        FB_CHECK_LAUNCH();
        sol[l] = Prec<T>::x(L);
        break;
      }
      case FB_COARSE_SMOOTHER:
        FB_TRY(presmooth<T>(m, l, b, bn, l == 0 || nu < 2, &sol[l]));
        break;
      case FB_COARSE_PCG: {
        T* w;
        if constexpr (std::is_same<T, double>::value) w = m->cg64; else w = m->cg32;
        const uint32_t nc = L.n;
        k_coarse_cg<T, 512><<<1, 512, 0, m->stream>>>(m->coarse_csr.view(!std::is_same<T, double>::value), b,
                                                      Prec<T>::x(L), w, w + nc, w + 2 * uint64_t(nc), L.mask, nc, 100);
        m->launches++;
        FB_CHECK_LAUNCH();
        sol[l] = Prec<T>::x(L);
        break;
      }
      case FB_COARSE_NONE:
      default:
        k_copy_masked<T><<<ew_grid(L.n), 256, 0, m->stream>>>(Prec<T>::x(L), b, L.mask, L.n);
        m->launches++;
        FB_CHECK_LAUNCH();
        sol[l] = Prec<T>::x(L);
        break;
    }
  }
  // ---- ascent (multigrid.hpp:1843-2000)
  for (int l = std::min(nl - 2, lc - 1); l >= 0; --l) {
    Level& L = m->L[l];
    const T* b = (l == 0) ? rhs_top : Prec<T>::rhs(L);
    T* cur = sol[l];
    T* oth = (cur == Prec<T>::x(L)) ? Prec<T>::y(L) : Prec<T>::x(L);
    EpiProlong<T> ep{cur, L.mask};
    FB_TRY(prol_T<T>(m, l, sol[l + 1], ep));
    T* s0 = cur;
    double* dn = &m->sc->lvl[2 * l + 1];
    for (int it = 0; it < nu; ++it) {
      if (it == 0) {
        EpiJacobi<T, true> e{cur, b, Prec<T>::invd(L), oth, nullptr, L.mask, nullptr, omega};
        FB_TRY(spmv_L<T>(m, L, cur, e, dn));
        if (nu == 1) {
          k_skip_fix<T><<<ew_grid(L.n), 256, 0, m->stream>>>(oth, s0, dn, L.n);
          m->launches++;
          FB_CHECK_LAUNCH();
        }
      } else if (l == 0 && it == nu - 1 && m->top_dot) {
        // the result is z: form PCG's r . z (rhs = r, or its FP32 copy in the mixed form) here
        EpiJacobi<T, false, true> e{cur, b, Prec<T>::invd(L), oth, s0, L.mask, dn, omega};
        FB_TRY(spmv_L<T>(m, L, cur, e, &m->sc->rz));
      } else {
        EpiJacobi<T, false> e{cur, b, Prec<T>::invd(L), oth, s0, L.mask, dn, omega};
        FB_TRY(spmv_L<T>(m, L, cur, e, nullptr));
      }
      std::swap(cur, oth);
    }
    sol[l] = cur;
  }
  *out_top = sol[0];
  return FB_OK;
}

// ------------------------------------------------------------------ F and W cycles, adaptive CGC
// MultiGrid::_apply_cycle_f / _apply_cycle_w (multigrid.hpp:1354-1519) built from the same
// fused pieces as the V-cycle: restriction from a level with or without its pre-smoothing
// (_apply_rest), prolongation up to a level with or without its post-smoothing (_apply_prol),
// with the fixed or adaptive coarse-grid correction, and the peak smoother (_apply_smooth_peak:
// the level's Richardson smoother on its defect, i.e. nu Jacobi steps from the current
// iterate, then the defect again). sol[l] tracks which ping-pong buffer holds level l's iterate.
template<typename T>
struct Cycle {
  fb_mg* m;
  const T* rhs_top;
  const double* rhs_top_sumsq;
  std::vector<T*> sol;
  int nl, nu;
  T omega;
  const T* rhs(int l) { return l == 0 ? rhs_top : Prec<T>::rhs(m->L[l]); }
  const double* bnorm(int l) { return l == 0 ? rhs_top_sumsq : &m->sc->lvl[2 * l]; }
  T* other(int l, T* cur) { Level& L = m->L[l]; return cur == Prec<T>::x(L) ? Prec<T>::y(L) : Prec<T>::x(L); }

  int defect(int l) {
    Level& L = m->L[l];
    EpiDefect<T, false, false> ed{Prec<T>::def(L), rhs(l), L.mask, nullptr};
    return spmv_L<T>(m, L, sol[l], ed, nullptr);
  }
  // nu Jacobi steps from sol[l] (the post-smoother on the defect equation): the first step
  // reduces the defect norm its successors test (the Richardson smoother's initial-norm test)
  int smooth_from(int l) {
    Level& L = m->L[l];
    T* cur = sol[l];
    T* oth = other(l, cur);
    T* s0 = cur;
    double* dn = &m->sc->lvl[2 * l + 1];
    for (int it = 0; it < nu; ++it) {
      if (it == 0) {
        EpiJacobi<T, true> e{cur, rhs(l), Prec<T>::invd(L), oth, nullptr, L.mask, nullptr, omega};
        FB_TRY(spmv_L<T>(m, L, cur, e, dn));
        if (nu == 1) {
          k_skip_fix<T><<<ew_grid(L.n), 256, 0, m->stream>>>(oth, s0, dn, L.n);
          m->launches++;
          FB_CHECK_LAUNCH();
        }
      } else {
        EpiJacobi<T, false> e{cur, rhs(l), Prec<T>::invd(L), oth, s0, L.mask, dn, omega};
        FB_TRY(spmv_L<T>(m, L, cur, e, nullptr));
      }
      std::swap(cur, oth);
    }
    sol[l] = cur;
    return FB_OK;
  }
  int rest(int cur, bool cur_smooth) {
    for (int i = cur; i + 1 < nl; ++i) {
      Level& L = m->L[i];
      Level& C = m->L[i + 1];
      if (cur_smooth || i > cur) {
        const bool need_s1 = (i == 0) ? !m->top_s1 : nu < 2;
        FB_TRY(presmooth<T>(m, i, rhs(i), bnorm(i), need_s1, &sol[i]));
        FB_TRY(defect(i));
      }
      const bool coarsest_next = (i + 2 == nl);
      T* s1 = nullptr;
      if (nu >= 2 && (!coarsest_next || m->cfg.coarse == FB_COARSE_SMOOTHER)) s1 = Prec<T>::x(C);
      EpiRestrict<T> er{Prec<T>::rhs(C), s1, Prec<T>::invd(C), C.mask, omega};
      FB_TRY(rest_T<T>(m, i, Prec<T>::def(L), er, &m->sc->lvl[2 * (i + 1)]));
    }
    return FB_OK;
  }
  int coarse() {
    const int l = nl - 1;
    Level& L = m->L[l];
    const T* b = rhs(l);
    switch (m->cfg.coarse) {
      case FB_COARSE_DIRECT: {
        const T* cinv;
        if constexpr (std::is_same<T, double>::value) cinv = m->cinv64; else cinv = m->cinv32;
        k_dense_solve<T><<<grid_for(uint64_t(L.n) * 32, 256), 256, 0, m->stream>>>(Prec<T>::x(L), cinv, b, L.n);
        m->launches++;
        FB_CHECK_LAUNCH();
        sol[l] = Prec<T>::x(L);
        break;
      }
      case FB_COARSE_SMOOTHER:
        FB_TRY(presmooth<T>(m, l, b, bnorm(l), l == 0 || nu < 2, &sol[l]));
        break;
      case FB_COARSE_PCG: {
        T* w;
        if constexpr (std::is_same<T, double>::value) w = m->cg64; else w = m->cg32;
        const uint32_t nc = L.n;
        k_coarse_cg<T, 512><<<1, 512, 0, m->stream>>>(m->coarse_csr.view(!std::is_same<T, double>::value), b,
                                                      Prec<T>::x(L), w, w + nc, w + 2 * uint64_t(nc), L.mask, nc, 100);
        m->launches++;
        FB_CHECK_LAUNCH();
        sol[l] = Prec<T>::x(L);
        break;
      }
      case FB_COARSE_NONE:
      default:
        k_copy_masked<T><<<ew_grid(L.n), 256, 0, m->stream>>>(Prec<T>::x(L), b, L.mask, L.n);
        m->launches++;
        FB_CHECK_LAUNCH();
        sol[l] = Prec<T>::x(L);
        break;
    }
    return FB_OK;
  }
  int prol(int cur, bool cur_smooth) {
    for (int i = nl - 2; i >= cur; --i) {
      Level& L = m->L[i];
      if (m->cfg.adapt_cgc == FB_CGC_FIXED) {
        EpiProlong<T> ep{sol[i], L.mask};
        FB_TRY(prol_T<T>(m, i, sol[i + 1], ep));
      } else {
        // cor = filter_cor(P x_c); tmp = filter_def(A cor); omega from the level's defect
        EpiFiltered<T> ec{Prec<T>::cor(L), L.mask};
        FB_TRY(prol_T<T>(m, i, sol[i + 1], ec));
        EpiFiltered<T> et{Prec<T>::tmp(L), L.mask};
        FB_TRY(spmv_L<T>(m, L, (const T*)Prec<T>::cor(L), et, nullptr));
        double* om = &m->sc->tmp[1];
        k_cgc_omega<T><<<kRedBlocks, 256, 0, m->stream>>>(Prec<T>::def(L), Prec<T>::cor(L), Prec<T>::tmp(L), L.n,
                                                          m->cfg.adapt_cgc == FB_CGC_MIN_DEFECT ? 1 : 0, m->ws,
                                                          m->counter, om);
        k_cgc_update<T><<<ew_grid(L.n), 256, 0, m->stream>>>(sol[i], Prec<T>::cor(L), om, L.n);
        m->launches += 2;
        FB_CHECK_LAUNCH();
      }
      // post-smoothing; the defect it starts from (rhs - A sol) is formed by its first step,
      // which equals def - omega * tmp of the adaptive correction up to rounding
      if (cur_smooth || i > cur) FB_TRY(smooth_from(i));
    }
    return FB_OK;
  }
  int peak(int l) {
    FB_TRY(smooth_from(l));
    return defect(l);
  }
};

template<typename T>
static int mgcycle(fb_mg* m, const T* rhs_top, const double* rhs_top_sumsq, T** out_top) {
  Cycle<T> c;
  c.m = m; c.rhs_top = rhs_top; c.rhs_top_sumsq = rhs_top_sumsq;
  c.nl = (int)m->L.size(); c.nu = m->cfg.nu; c.omega = T(m->cfg.omega_rich);
  c.sol.assign(c.nl, nullptr);
  const int last = c.nl - 1;
  FB_TRY(c.rest(0, true));
  if (m->cfg.cycle == FB_CYCLE_F) {
    for (int pk = last - 1; pk > 0; --pk) {
      FB_TRY(c.coarse());
      FB_TRY(c.prol(pk, false));
      FB_TRY(c.peak(pk));
      FB_TRY(c.rest(pk, false));
    }
    FB_TRY(c.coarse());
  } else if (m->cfg.cycle == FB_CYCLE_W) {
    FB_TRY(c.coarse());
    // 2^(levels-1) coarse solves; the next peak is the lowest level above the coarse one whose
    // counter is 0 (multigrid.hpp:1430-1500)
    std::vector<int> cnt(c.nl, 0);
    const int num_cgs = 1 << last;
    for (int cgs = 1; cgs < num_cgs; ++cgs) {
      int pk = last;
      while (pk > 0)
        if (cnt[--pk] == 0) break;
      for (int i = last - 1; i > pk; --i) cnt[i] = 0;
      ++cnt[pk];
      FB_TRY(c.prol(pk, false));
      FB_TRY(c.peak(pk));
      FB_TRY(c.rest(pk, false));
      FB_TRY(c.coarse());
    }
  } else {
    FB_TRY(c.coarse());
  }
  FB_TRY(c.prol(0, true));
  *out_top = c.sol[0];
  return FB_OK;
}

// the V-cycle with the fixed correction has its own driver (fused coarse end, r.z inside)
template<typename T>
static int mg_apply(fb_mg* m, const T* rhs_top, const double* rhs_top_sumsq, T** out_top) {
  if (m->cfg.cycle == FB_CYCLE_V && m->cfg.adapt_cgc == FB_CGC_FIXED) return vcycle<T>(m, rhs_top, rhs_top_sumsq, out_top);
  return mgcycle<T>(m, rhs_top, rhs_top_sumsq, out_top);
}

// ------------------------------------------------------------------ stopping logic
// IterativeSolver defaults and tests (kernel/solver/iterative.hpp:216-235, 490-505, 744-832)
struct Stop {
  double tol_rel, tol_abs, tol_abs_low = 0.0, div_rel, div_abs, def_init = 0.0;
  int max_iter;
  Stop(double tr, int mi) : tol_rel(tr), max_iter(mi) {
    const double e = eps_of<double>();
    tol_abs = 1.0 / (e * e); div_rel = 1.0 / e; div_abs = 1.0 / (e * e);
  }
  int initial(double d) {
    def_init = d;
    if (!std::isfinite(d)) return 3;
    if (d <= eps_of<double>() * eps_of<double>()) return 2;
    return 1;
  }
  int analyse(int it, double d) const {
    if (!std::isfinite(d)) return 3;
    if (d > div_abs || d > div_rel * def_init) return 4;
    if ((d <= tol_abs) && ((d <= tol_rel * def_init) || (d <= tol_abs_low))) return 2;
    if (it >= max_iter) return 5;
    return 1;
  }
};

// ------------------------------------------------------------------ solver bodies
// PCG outer with nu >= 2 on two or more levels: the PCG update kernel also forms the first
// pre-smoothing step of the next V-cycle on the finest level (k_jacobi0 is not launched there)
static bool fuse_s1(const fb_mg* m) {
  return m->cfg.outer == FB_OUTER_PCG && m->cfg.nu >= 2 && m->L.size() > 1;
}
// ... and its last post-smoothing step forms r . z (z = that step's result, r = the V-cycle's
// right-hand side: the outer defect, or its FP32 copy in the mixed forms)
static bool fuse_dot(const fb_mg* m) {
  return m->cfg.outer == FB_OUTER_PCG && m->cfg.nu >= 2 && m->L.size() > 1 && !(m->cfg.flags & FB_FLAG_NO_DOT_FUSION) &&
         m->cfg.cycle == FB_CYCLE_V && m->cfg.adapt_cgc == FB_CGC_FIXED;
}

// outer defect r = filter_def(b - A x), ||r||^2, FP32 copy for the mixed V-cycle
static int outer_defect(fb_mg* m) {
  Level& L = m->L[0];
  if (m->cfg.precision == FB_PREC_F64) {
    EpiDefect<double, true, false> e{m->r, m->bb, L.mask, nullptr};
    return spmv_L<double>(m, L, (const double*)m->xb, e, &m->sc->rr);
  }
  EpiDefect<double, true, true> e{m->r, m->bb, L.mask, m->r32};
  return spmv_L<double>(m, L, (const double*)m->xb, e, &m->sc->rr);
}

// z-like output of the preconditioner (FP64 or FP32 buffer)
static int precond(fb_mg* m, const void** z_out) {
  if (m->cfg.precision == FB_PREC_F64) {
    double* z = nullptr;
    FB_TRY(mg_apply<double>(m, m->r, &m->sc->rr, &z));
    *z_out = z;
  } else {
    float* z = nullptr;
    FB_TRY(mg_apply<float>(m, m->r32, &m->sc->rr, &z));
    *z_out = z;
  }
  return FB_OK;
}

// one outer iteration after a successful stopping test; ends with ||r||^2 copied to the host
// iteration j (from 1) of the outer solver; PCG's direction buffers alternate with j's parity
static int body(fb_mg* m, int j) {
  const uint32_t n = m->L[0].n;
  const bool low = m->cfg.precision != FB_PREC_F64;
  const void* z = nullptr;
  m->top_s1 = fuse_s1(m);
  m->top_dot = fuse_dot(m);
  const int pst = precond(m, &z);
  m->top_s1 = false;
  const bool dot_done = m->top_dot;
  m->top_dot = false;
  FB_TRY(pst);
  if (m->cfg.outer == FB_OUTER_PCG) {
    // gamma' = r . z ; p = z + beta p ; q = A p ; x, r update
    if (!dot_done) {
      if (low) FB_CUDA(launch_pdl(m->stream, k_dot_rz<float>, dim3(occupancy_grid((const void*)k_dot_rz<float>, n / 32 + 1)),
                                  dim3(256), 0, (const double*)m->r, (const float*)z, n, m->ws, m->counter, &m->sc->rz));
      else     FB_CUDA(launch_pdl(m->stream, k_dot_rz<double>, dim3(occupancy_grid((const void*)k_dot_rz<double>, n / 32 + 1)),
                                  dim3(256), 0, (const double*)m->r, (const double*)z, n, m->ws, m->counter, &m->sc->rz));
      m->launches++;
      FB_CHECK_LAUNCH();
    }
    const bool p32 = pcg_p32(m);
    const bool odd = (j & 1) != 0;
    float* pf_out = odd ? m->p32b : m->p32;
    float* pf_in = odd ? m->p32 : m->p32b;
    double* pd_out = odd ? m->pb : m->p;
    double* pd_in = odd ? m->p : m->pb;
    const dim3 eg(ew_grid(n));
    if (p32) {
      if (odd) FB_CUDA(launch_pdl(m->stream, k_pcg_dir2<float, float, false>, eg, dim3(256), 0, pf_out, (const float*)pf_in,
                                  m->xb, (const float*)z, m->sc, n));
      else     FB_CUDA(launch_pdl(m->stream, k_pcg_dir2<float, float, true>, eg, dim3(256), 0, pf_out, (const float*)pf_in,
                                  m->xb, (const float*)z, m->sc, n));
    } else if (low) {
      if (odd) FB_CUDA(launch_pdl(m->stream, k_pcg_dir2<float, double, false>, eg, dim3(256), 0, pd_out,
                                  (const double*)pd_in, m->xb, (const float*)z, m->sc, n));
      else     FB_CUDA(launch_pdl(m->stream, k_pcg_dir2<float, double, true>, eg, dim3(256), 0, pd_out,
                                  (const double*)pd_in, m->xb, (const float*)z, m->sc, n));
    } else {
      if (odd) FB_CUDA(launch_pdl(m->stream, k_pcg_dir2<double, double, false>, eg, dim3(256), 0, pd_out,
                                  (const double*)pd_in, m->xb, (const double*)z, m->sc, n));
      else     FB_CUDA(launch_pdl(m->stream, k_pcg_dir2<double, double, true>, eg, dim3(256), 0, pd_out,
                                  (const double*)pd_in, m->xb, (const double*)z, m->sc, n));
    }
    m->launches++;
    FB_CHECK_LAUNCH();
    if (p32) {
      FB_TRY(pcgq_p32(m, &m->sc->qp, pf_out));
    } else {
      EpiPcgQ<double> eq{m->q, pd_out, m->L[0].mask};
      FB_TRY(spmv_L<double>(m, m->L[0], (const double*)pd_out, eq, &m->sc->qp));
    }
    Level& L0 = m->L[0];
    const bool fs = fuse_s1(m);
    if (low) FB_CUDA(launch_pdl(m->stream, k_pcg_update<true>, dim3(occupancy_grid((const void*)k_pcg_update<true>, n / 32 + 1)),
                                dim3(256), 0, m->r, m->r32, (const double*)m->q, m->sc, n,
                                m->ws, m->counter, &m->sc->rr, fs ? (void*)L0.x32 : nullptr, (const void*)L0.invd32,
                                (const uint32_t*)L0.mask, m->cfg.omega_rich));
    else     FB_CUDA(launch_pdl(m->stream, k_pcg_update<false>, dim3(occupancy_grid((const void*)k_pcg_update<false>, n / 32 + 1)),
                                dim3(256), 0, m->r, m->r32, (const double*)m->q, m->sc, n,
                                m->ws, m->counter, &m->sc->rr, fs ? (void*)L0.x64 : nullptr, (const void*)L0.invd64,
                                (const uint32_t*)L0.mask, m->cfg.omega_rich));
    m->launches++;
    FB_CHECK_LAUNCH();
  } else {
    if (low) k_rich_update<float><<<ew_grid(n), 256, 0, m->stream>>>(m->xb, (const float*)z, m->cfg.omega_outer, n);
    else     k_rich_update<double><<<ew_grid(n), 256, 0, m->stream>>>(m->xb, (const double*)z, m->cfg.omega_outer, n);
    m->launches++;
    FB_CHECK_LAUNCH();
    FB_TRY(outer_defect(m));
  }
  FB_CUDA(cudaMemcpyAsync(m->host_rr, &m->sc->rr, kHostScalarBytes, cudaMemcpyDeviceToHost, m->stream));
  return FB_OK;
}

static int run_body(fb_mg* m, int j) {
  if (!m->cfg.use_graphs || debug_enabled()) return body(m, j);
  // one graph per parity of j (the direction buffers alternate)
  const int par = j & 1;
  const int key = ((m->cfg.cycle * 4 + m->cfg.adapt_cgc) * 16 + m->cfg.flags) * 256 + m->cfg.format * 64 +
                  m->cfg.precision * 16 + m->cfg.outer * 4 + m->cfg.coarse;
  cudaGraphExec_t& gb = m->g_body[par];
  if (!gb || m->g_body_key[par] != key) {
    if (gb) { cudaGraphExecDestroy(gb); gb = nullptr; }
    cudaGraph_t g = nullptr;
    FB_CUDA(cudaStreamBeginCapture(m->stream, cudaStreamCaptureModeThreadLocal));
    const int before = m->launches;
    int st = body(m, j);
    cudaError_t e = cudaStreamEndCapture(m->stream, &g);
    m->body_launches = m->launches - before;
    m->launches = before;
    if (st != FB_OK) { if (g) cudaGraphDestroy(g); return st; }
    if (e != cudaSuccess) return FB_ERR_CUDA;
    e = cudaGraphInstantiate(&gb, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) { gb = nullptr; return FB_ERR_CUDA; }
    m->g_body_key[par] = key;
  }
  m->launches += m->body_launches;
  FB_CUDA(cudaGraphLaunch(gb, m->stream));
  return FB_OK;
}

static int ensure_vectors(fb_mg* m, int prec) {
  if (m->prec_built == prec) return FB_OK;
  const int nl = (int)m->L.size();
  const bool low = prec != FB_PREC_F64;
  for (int l = 0; l < nl; ++l) {
    Level& L = m->L[l];
    if (!low && !L.x64) {
      if (l > 0) FB_TRY(dalloc(m, &L.rhs64, L.n));
      FB_TRY(dalloc(m, &L.x64, L.n)); FB_TRY(dalloc(m, &L.y64, L.n)); FB_TRY(dalloc(m, &L.def64, L.n));
    }
    if (low && !L.x32) {
      if (l > 0) FB_TRY(dalloc(m, &L.rhs32, L.n));
      FB_TRY(dalloc(m, &L.x32, L.n)); FB_TRY(dalloc(m, &L.y32, L.n)); FB_TRY(dalloc(m, &L.def32, L.n));
    }
    if (!L.invd64) FB_TRY(dalloc(m, &L.invd64, L.n));
    if (low && !L.invd32) FB_TRY(dalloc(m, &L.invd32, L.n));
    if (m->cfg.adapt_cgc != FB_CGC_FIXED) {
      if (!low && !L.cor64) { FB_TRY(dalloc(m, &L.cor64, L.n)); FB_TRY(dalloc(m, &L.tmp64, L.n)); }
      if (low && !L.cor32) { FB_TRY(dalloc(m, &L.cor32, L.n)); FB_TRY(dalloc(m, &L.tmp32, L.n)); }
    }
    k_invdiag<<<ew_grid(L.n), 256, 0, m->stream>>>(L.invd64, low ? L.invd32 : nullptr, L.diag, m->cfg.omega_jac, L.n);
    FB_CHECK_LAUNCH();
    if (low) {
      if (!L.P.v32 && L.P.nnz) {
        FB_TRY(dalloc(m, &L.P.v32, L.P.nnz)); FB_TRY(dalloc(m, &L.R.v32, L.R.nnz));
        k_cvt<float, double><<<ew_grid(L.P.nnz), 256, 0, m->stream>>>(L.P.v32, L.P.v64, L.P.nnz);
        k_cvt<float, double><<<ew_grid(L.R.nnz), 256, 0, m->stream>>>(L.R.v32, L.R.v64, L.R.nnz);
        FB_CHECK_LAUNCH();
      }
      const bool mf = m->cfg.format == FB_FORMAT_MATFREE && L.mf;
      const bool need_st = m->cfg.format != FB_FORMAT_SELL && L.St.S && !mf;
      const bool need_sell = !mf && !need_st;
      if (need_st && prec == FB_PREC_F32 && !L.St.v32) {
        const uint64_t np = uint64_t(L.St.nchunks) * ((L.St.S + 1) / 2) * 32 * 2;
        FB_TRY(dalloc(m, &L.St.v32, np));
        k_stencil_pack<float><<<ew_grid(np), 256, 0, m->stream>>>(L.St.v32, L.St.v64, L.St.nchunks, L.St.S, 1.0);
        FB_CHECK_LAUNCH();
      }
      if (need_st && prec == FB_PREC_F16 && !L.St.v16) {
        const uint64_t ns = uint64_t(L.St.nchunks) * L.St.S * 32;
        unsigned long long* dmax = nullptr;
        FB_TRY(dalloc(m, &dmax, 1));
        FB_CUDA(cudaMemsetAsync(dmax, 0, sizeof(unsigned long long), m->stream));
        k_absmax<<<ew_grid(ns), 256, 0, m->stream>>>(L.St.v64, ns, dmax);
        FB_CHECK_LAUNCH();
        unsigned long long hm = 0;
        FB_CUDA(cudaMemcpyAsync(&hm, dmax, sizeof(hm), cudaMemcpyDeviceToHost, m->stream));
        FB_CUDA(cudaStreamSynchronize(m->stream));
        double amax;
        std::memcpy(&amax, &hm, sizeof(double));
        L.St.scale16 = float(amax > 0.0 ? amax / 16384.0 : 1.0);
        const uint64_t np = uint64_t(L.St.nchunks) * ((L.St.S + 3) / 4) * 32 * 4;
        FB_TRY(dalloc(m, &L.St.v16, np));
        k_stencil_pack<__half><<<ew_grid(np), 256, 0, m->stream>>>(L.St.v16, L.St.v64, L.St.nchunks, L.St.S,
                                                                     1.0 / double(L.St.scale16));
        FB_CHECK_LAUNCH();
      }
      if (need_sell && prec == FB_PREC_F32 && !L.A.v32) {
        FB_TRY(dalloc(m, &L.A.v32, L.A.nent));
        k_cvt<float, double><<<ew_grid(L.A.nent), 256, 0, m->stream>>>(L.A.v32, L.A.v64, L.A.nent);
        FB_CHECK_LAUNCH();
      }
      if (need_sell && prec == FB_PREC_F16 && !L.A.v16) {
        // per-level scale: the largest magnitude maps to 2^14 (headroom below 65504)
        unsigned long long* dmax = nullptr;
        FB_TRY(dalloc(m, &dmax, 1));
        FB_CUDA(cudaMemsetAsync(dmax, 0, sizeof(unsigned long long), m->stream));
        k_absmax<<<ew_grid(L.A.nent), 256, 0, m->stream>>>(L.A.v64, L.A.nent, dmax);
        FB_CHECK_LAUNCH();
        unsigned long long hm = 0;
        FB_CUDA(cudaMemcpyAsync(&hm, dmax, sizeof(hm), cudaMemcpyDeviceToHost, m->stream));
        FB_CUDA(cudaStreamSynchronize(m->stream));
        double amax;
        std::memcpy(&amax, &hm, sizeof(double));
        const double scale = amax > 0.0 ? amax / 16384.0 : 1.0;
        L.A.scale16 = float(scale);
        FB_TRY(dalloc(m, &L.A.v16, L.A.nent));
        k_quant16_sell<<<ew_grid(uint64_t(L.A.nchunks) * 32), 256, 0, m->stream>>>(
            L.A.v16, L.A.v64, 1.0 / double(L.A.scale16), L.A.cs, L.A.cl, L.A.nchunks);
        FB_CHECK_LAUNCH();
      }
    }
  }
  if (m->coarse_csr.rp) {
    const uint64_t nc = m->coarse_csr.rows;
    if (!low && !m->cg64) FB_TRY(dalloc(m, &m->cg64, 3 * nc));
    if (low && !m->cg32) FB_TRY(dalloc(m, &m->cg32, 3 * nc));
    if (low && !m->coarse_csr.v32) {
      FB_TRY(dalloc(m, &m->coarse_csr.v32, m->coarse_csr.nnz));
      k_cvt<float, double><<<ew_grid(m->coarse_csr.nnz), 256, 0, m->stream>>>(m->coarse_csr.v32, m->coarse_csr.v64, m->coarse_csr.nnz);
      FB_CHECK_LAUNCH();
    }
  }
  if (low && m->cinv64 && !m->cinv32) {
    FB_TRY(dalloc(m, &m->cinv32, uint64_t(m->nc) * m->nc));
    k_cvt<float, double><<<ew_grid(uint64_t(m->nc) * m->nc), 256, 0, m->stream>>>(m->cinv32, m->cinv64, uint64_t(m->nc) * m->nc);
    FB_CHECK_LAUNCH();
  }
  const uint32_t n = m->L[0].n;
  if (!m->r) {
    FB_TRY(dalloc(m, &m->r, n)); FB_TRY(dalloc(m, &m->p, n)); FB_TRY(dalloc(m, &m->q, n));
    FB_TRY(dalloc(m, &m->pb, n));
    FB_TRY(dalloc(m, &m->p32, n)); FB_TRY(dalloc(m, &m->p32b, n));
    FB_TRY(dalloc(m, &m->xb, n)); FB_TRY(dalloc(m, &m->bb, n));
  }
  if (low && !m->r32) FB_TRY(dalloc(m, &m->r32, n));
  m->prec_built = prec;
  FB_CUDA(cudaStreamSynchronize(m->stream));
  return FB_OK;
}

// ------------------------------------------------------------------ setup: CSR -> SELL
// SELL-C-sigma with C = 32: rows sorted by decreasing length inside windows of sigma rows
int upload_sell(fb_mg* m, DevSell& S, const HostCsr& A, int sigma) {
  const uint64_t n = A.rows;
  if (n > 0xffffffffull) return FB_ERR_INVALID;
  S.rows = uint32_t(n); S.cols = uint32_t(A.cols); S.nnz = A.rp[n];
  S.nchunks = uint32_t((n + 31) / 32);
  std::vector<uint32_t> perm(n);
  std::iota(perm.begin(), perm.end(), 0u);
  if (sigma > 1) {
    for (uint64_t w = 0; w < n; w += sigma) {
      const uint64_t e = std::min<uint64_t>(n, w + sigma);
      std::stable_sort(perm.begin() + w, perm.begin() + e, [&](uint32_t a, uint32_t b) {
        return (A.rp[a + 1] - A.rp[a]) > (A.rp[b + 1] - A.rp[b]);
      });
    }
  }
  std::vector<uint32_t> cs(S.nchunks + 1, 0), cl(S.nchunks, 0);
  for (uint32_t c = 0; c < S.nchunks; ++c) {
    uint32_t mx = 0;
    for (uint32_t t = 0; t < 32; ++t) {
      const uint64_t sr = uint64_t(c) * 32 + t;
      if (sr < n) mx = std::max<uint32_t>(mx, uint32_t(A.rp[perm[sr] + 1] - A.rp[perm[sr]]));
    }
    cl[c] = mx;
    const uint64_t nx = uint64_t(cs[c]) + uint64_t(mx) * 32;
    if (nx > 0xffffffffull) return FB_ERR_INVALID;
    cs[c + 1] = uint32_t(nx);
  }
  S.nent = cs[S.nchunks];
  std::vector<uint32_t> col(S.nent, 0);
  std::vector<double> val(S.nent, 0.0);
  for (uint64_t sr = 0; sr < n; ++sr) {
    const uint32_t row = perm[sr];
    const uint32_t c = uint32_t(sr / 32), t = uint32_t(sr % 32);
    uint32_t j = 0;
    for (uint64_t k = A.rp[row]; k < A.rp[row + 1]; ++k, ++j) {
      col[cs[c] + uint64_t(j) * 32 + t] = A.ci[k];
      val[cs[c] + uint64_t(j) * 32 + t] = A.va[k];
    }
    // padding: column of the row itself (keeps x loads in the row's neighbourhood), value 0
    for (; j < cl[c]; ++j) col[cs[c] + uint64_t(j) * 32 + t] = row < A.cols ? row : 0;
  }
  FB_TRY(dupload(m, &S.cs, cs.data(), cs.size()));
  FB_TRY(dupload(m, &S.cl, cl.data(), cl.size()));
  FB_TRY(dupload(m, &S.col, col.data(), col.size()));
  FB_TRY(dupload(m, &S.v64, val.data(), val.size()));
  {
    std::vector<uint32_t> rl(n);
    for (uint64_t i = 0; i < n; ++i) rl[i] = uint32_t(A.rp[i + 1] - A.rp[i]);
    FB_TRY(dupload(m, &S.rl, rl.data(), rl.size()));
  }
  if (sigma > 1) FB_TRY(dupload(m, &S.perm, perm.data(), perm.size()));
  return FB_OK;
}

int upload_csr(fb_mg* m, DevCsr& D, const HostCsr& A) {
  if (A.rows > 0xffffffffull || A.rp[A.rows] > 0xffffffffull) return FB_ERR_INVALID;
  D.rows = uint32_t(A.rows); D.cols = uint32_t(A.cols); D.nnz = A.rp[A.rows];
  std::vector<uint32_t> rp(A.rp.begin(), A.rp.end());
  FB_TRY(dupload(m, &D.rp, rp.data(), rp.size()));
  FB_TRY(dupload(m, &D.col, A.ci.data(), A.ci.size()));
  FB_TRY(dupload(m, &D.v64, A.va.data(), A.va.size()));
  return FB_OK;
}

int upload_coarse_csr(fb_mg* m, const HostCsr& A) {
  if (A.rows > 65536) return FB_OK;  // the single-CTA coarse CG is offered for small coarse levels only
  return upload_csr(m, m->coarse_csr, A);
}

int upload_filter(fb_mg* m, Level& L, const std::vector<uint32_t>& f) {
  std::vector<uint32_t> mask((L.n + 31) / 32, 0u);
  for (uint32_t i : f) {
    if (i >= L.n) return FB_ERR_INVALID;
    mask[i >> 5] |= 1u << (i & 31);
  }
  FB_TRY(dupload(m, &L.mask, mask.data(), mask.size()));
  FB_TRY(dupload(m, &L.filt, f.data(), f.size()));
  L.nfilt = uint32_t(f.size());
  return FB_OK;
}

// dense inverse of the filtered coarse matrix (Dirichlet rows/columns -> 0), Gauss-Jordan
// with partial pivoting in FP64 on the host (setup only)
int build_coarse_inverse(fb_mg* m, const HostCsr& A, const std::vector<uint32_t>& filt) {
  const uint64_t n = A.rows;
  if (n > 4096) { m->nc = 0; return FB_OK; }  // direct coarse solve limited to small coarse levels
  std::vector<char> dir(n, 0);
  for (auto i : filt) dir[i] = 1;
  std::vector<double> a(n * n, 0.0), inv(n * n, 0.0);
  for (uint64_t i = 0; i < n; ++i) {
    inv[i * n + i] = 1.0;
    if (dir[i]) { a[i * n + i] = 1.0; continue; }
    for (uint64_t k = A.rp[i]; k < A.rp[i + 1]; ++k)
      if (!dir[A.ci[k]]) a[i * n + A.ci[k]] = A.va[k];
  }
  for (uint64_t c = 0; c < n; ++c) {
    uint64_t p = c;
    for (uint64_t i = c + 1; i < n; ++i) if (std::fabs(a[i * n + c]) > std::fabs(a[p * n + c])) p = i;
    if (a[p * n + c] == 0.0) return FB_ERR_INVALID;  // singular coarse matrix
    if (p != c) for (uint64_t j = 0; j < n; ++j) { std::swap(a[c * n + j], a[p * n + j]); std::swap(inv[c * n + j], inv[p * n + j]); }
    const double d = 1.0 / a[c * n + c];
    for (uint64_t j = 0; j < n; ++j) { a[c * n + j] *= d; inv[c * n + j] *= d; }
    for (uint64_t i = 0; i < n; ++i) {
      if (i == c) continue;
      const double f = a[i * n + c];
      if (f == 0.0) continue;
      for (uint64_t j = 0; j < n; ++j) { a[i * n + j] -= f * a[c * n + j]; inv[i * n + j] -= f * inv[c * n + j]; }
    }
  }
  for (uint64_t i = 0; i < n; ++i)
    for (uint64_t j = 0; j < n; ++j)
      if (dir[i] || dir[j]) inv[i * n + j] = 0.0;
  m->nc = uint32_t(n);
  FB_TRY(dupload(m, &m->cinv64, inv.data(), inv.size()));
  return FB_OK;
}

int common_init(fb_mg* m) {
  FB_CUDA(cudaGetDevice(&m->device));
  FB_CUDA(cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking));
  FB_TRY(dalloc(m, &m->sc, 1));
  FB_CUDA(cudaMemsetAsync(m->sc, 0, sizeof(DevScalars), m->stream));
  FB_TRY(dalloc(m, &m->ws, 8192));
  FB_TRY(dalloc(m, &m->counter, 4));
  FB_CUDA(cudaMemsetAsync(m->counter, 0, 4 * sizeof(unsigned), m->stream));
  FB_TRY(dalloc(m, &m->dbg_err, 1));
  FB_CUDA(cudaMemsetAsync(m->dbg_err, 0, sizeof(unsigned long long), m->stream));
  m->kerr = &m->sc->kerr;
  m->inject = &m->sc->inject;
  FB_CUDA(cudaStreamSynchronize(m->stream));
  FB_CUDA(cudaMallocHost(&m->host_rr, sizeof(double) * 4));
  FB_CUDA(cudaEventCreate(&m->ev0));
  FB_CUDA(cudaEventCreate(&m->ev1));
  fb_solver_cfg_default(&m->cfg);
  return FB_OK;
}

__global__ void k_diag_sell(double* d, SellView A) {
  const uint32_t sr = blockIdx.x * blockDim.x + threadIdx.x;
  if (sr >= A.rows) return;
  const uint32_t c = sr / 32, t = sr % 32;
  const uint32_t row = A.perm ? A.perm[sr] : sr;
  double v = 0.0;
  const double* val = (const double*)A.val;
  for (uint32_t j = 0; j < A.cl[c]; ++j) {
    const uint32_t k = A.cs[c] + j * 32 + t;
    if (A.col[k] == row && val[k] != 0.0) { v = val[k]; break; }
  }
  d[row] = v;
}

int finish_levels(fb_mg* m) {
  // reduction partials: one per CTA of the largest reducing launch (3D-grid restriction)
  uint64_t need = 8192;
  for (auto& L : m->L)
    if (L.q1_transfer)
      need = std::max<uint64_t>(need, uint64_t((L.tr.Mc1 + 31) / 32) * ((L.tr.Mc1 + 7) / 8) * (L.tr.dim == 3 ? L.tr.Mc1 : 1));
  if (need > 8192) FB_TRY(dalloc(m, &m->ws, need));
  for (auto& L : m->L) {
    if (L.diag) continue;  // structured levels: formed from the row gather at creation
    FB_TRY(dalloc(m, &L.diag, L.n));
    k_diag_sell<<<grid_for(L.n, 256), 256, 0, m->stream>>>(L.diag, L.A.view(FB_PREC_F64));
    FB_CHECK_LAUNCH();
  }
  FB_CUDA(cudaStreamSynchronize(m->stream));
  return FB_OK;
}

// the kernel-wait flag as of the last read-back of the scalars
static bool host_kerr(const fb_mg* m) {
  unsigned f = 0;
  std::memcpy(&f, reinterpret_cast<const char*>(m->host_rr) + offsetof(DevScalars, kerr), sizeof(f));
  return f != 0;
}

// a bounded wait inside a staged kernel expired: report it (and clear the flag)
static int check_kernel_waits(fb_mg* m) {
  unsigned h = 0;
  FB_CUDA(cudaMemcpyAsync(&h, m->kerr, sizeof(h), cudaMemcpyDeviceToHost, m->stream));
  FB_CUDA(cudaStreamSynchronize(m->stream));
  if (!h) return FB_OK;
  FB_CUDA(cudaMemsetAsync(m->kerr, 0, sizeof(unsigned), m->stream));
  if (debug_enabled()) std::fprintf(stderr, "feat3_b200: staged kernel wait expired (code %u)\n", h);
  return FB_ERR_TIMEOUT;
}

// ------------------------------------------------------------------ solve
int solve_dev(fb_mg* m, const double* rhs, double* sol, double* hist, fb_solve_info* info, bool feat_io) {
  if (!m->configured) return FB_ERR_NOT_READY;
  FB_TRY(ensure_vectors(m, m->cfg.precision));
  const uint32_t n = m->L[0].n;
  cudaStream_t s = m->stream;
  const uint32_t* perm = feat_io ? m->feat_dof : nullptr;
  m->launches = 0;
  FB_CUDA(cudaEventRecord(m->ev0, s));
  if (perm) {
    FB_TRY(perm_to_lattice(m, m->bb, rhs, perm, n));
    FB_TRY(perm_to_lattice(m, m->xb, sol, perm, n));
  } else {
    FB_CUDA(cudaMemcpyAsync(m->bb, rhs, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
    FB_CUDA(cudaMemcpyAsync(m->xb, sol, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
  }
  // correct(): r = filter_def(b - A x) (pcg.hpp:158-172, richardson.hpp:174-185)
  FB_TRY(outer_defect(m));
  if (m->cfg.outer == FB_OUTER_PCG) {
    k_init_pcg<<<1, 1, 0, s>>>(m->sc);
    if (pcg_p32(m)) k_fill<float><<<ew_grid(n), 256, 0, s>>>(m->p32, 0.0f, n);
    else k_fill<double><<<ew_grid(n), 256, 0, s>>>(m->p, 0.0, n);
    m->launches += 2;
    FB_CHECK_LAUNCH();
    if (fuse_s1(m)) {
      // first pre-smoothing step of the first V-cycle (later ones come from k_pcg_update)
      Level& L0 = m->L[0];
      const double om = m->cfg.omega_rich;
      if (m->cfg.precision == FB_PREC_F64)
        k_jacobi0<double><<<ew_grid(n), 256, 0, s>>>(L0.x64, m->r, L0.invd64, L0.mask, &m->sc->rr, om, n);
      else
        k_jacobi0<float><<<ew_grid(n), 256, 0, s>>>(L0.x32, m->r32, L0.invd32, L0.mask, &m->sc->rr, float(om), n);
      m->launches++;
      FB_CHECK_LAUNCH();
    }
  }
  FB_CUDA(cudaMemcpyAsync(m->host_rr, &m->sc->rr, kHostScalarBytes, cudaMemcpyDeviceToHost, s));
  FB_CUDA(cudaStreamSynchronize(s));
  Stop st(m->cfg.tol_rel, m->cfg.max_iter);
  double d = std::sqrt(*m->host_rr);
  int status = st.initial(d);
  int it = 0;
  if (hist) hist[0] = d;
  // a staged kernel whose bounded wait expired has left rows unwritten: the solve stops at the
  // next read-back and returns FB_ERR_TIMEOUT (check_kernel_waits below)
  while (status == 1 && !host_kerr(m)) {
    FB_TRY(run_body(m, it + 1));
    FB_CUDA(cudaStreamSynchronize(s));
    ++it;
    d = std::sqrt(*m->host_rr);
    if (hist) hist[it] = d;
    status = st.analyse(it, d);
  }
  if (m->cfg.outer == FB_OUTER_PCG) {
    // after `it` iterations: p_it is in buffer it & 1; an even count also holds alpha_{it-1} p_{it-1}
    const bool odd = (it & 1) != 0;
    if (pcg_p32(m))
      k_pcg_finish2<float><<<ew_grid(n), 256, 0, s>>>(m->xb, m->p32b, odd ? m->p32b : m->p32, m->sc, n, odd ? 0 : 1);
    else
      k_pcg_finish2<double><<<ew_grid(n), 256, 0, s>>>(m->xb, m->pb, odd ? m->pb : m->p, m->sc, n, odd ? 0 : 1);
    m->launches++;
    FB_CHECK_LAUNCH();
  }
  if (perm) FB_TRY(perm_from_lattice(m, sol, m->xb, perm, n));
  else FB_CUDA(cudaMemcpyAsync(sol, m->xb, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
  FB_CUDA(cudaEventRecord(m->ev1, s));
  FB_CUDA(cudaEventSynchronize(m->ev1));
  FB_TRY(check_kernel_waits(m));
  if (check_enabled()) FB_TRY(check_self_checks(m));
  float ms = 0.0f;
  cudaEventElapsedTime(&ms, m->ev0, m->ev1);
  if (info) {
    info->status = status; info->iters = it; info->def_init = st.def_init; info->def_final = d;
    info->solve_ms = ms; info->kernel_launches = m->launches;
  }
  return FB_OK;
}

}  // namespace fb

using namespace fb;

// ====================================================================================== C-ABI
extern "C" {

void fb_solver_cfg_default(fb_solver_cfg* c) {
  if (!c) return;
  c->outer = FB_OUTER_PCG;
  c->nu = 4;
  c->omega_jac = 0.5;
  c->omega_rich = 1.0;
  c->omega_outer = 1.0;
  c->coarse = FB_COARSE_DIRECT;
  c->tol_rel = 1e-8;
  c->max_iter = 1000;
  c->precision = FB_PREC_F64;
  c->use_graphs = 1;
  c->format = FB_FORMAT_SELL;
  c->flags = 0;
  c->cycle = FB_CYCLE_V;
  c->adapt_cgc = FB_CGC_FIXED;
}

int fb_mg_configure(fb_mg* m, const fb_solver_cfg* c) {
  if (!m || !c) return FB_ERR_INVALID;
  if (c->nu < 1 || c->nu > 64 || c->max_iter < 0 || !(c->tol_rel >= 0.0) ||
      c->precision < 0 || c->precision > 2 || c->outer < 0 || c->outer > 1 || c->coarse < 0 || c->coarse > 3 ||
      c->format < 0 || c->format > 2 || c->cycle < 0 || c->cycle > 2 || c->adapt_cgc < 0 || c->adapt_cgc > 2 ||
      (c->flags & ~15))
    return FB_ERR_INVALID;
  if (c->coarse == FB_COARSE_PCG && !m->coarse_csr.rp) return FB_ERR_UNSUPPORTED;
  if (c->coarse == FB_COARSE_DIRECT && !m->cinv64) return FB_ERR_UNSUPPORTED;
  FB_CUDA(cudaSetDevice(m->device));
  // the assembled formats need the level matrices (and SELL the CSR transfers) of the large levels
  if (c->format != FB_FORMAT_MATFREE) FB_TRY(ensure_assembled(m, true, c->format == FB_FORMAT_SELL));
  m->cfg = *c;
  m->configured = true;
  for (int q = 0; q < 2; ++q)
    if (m->g_body[q]) { cudaGraphExecDestroy(m->g_body[q]); m->g_body[q] = nullptr; m->g_body_key[q] = -1; }
  m->prec_built = -1;
  return ensure_vectors(m, c->precision);
}

int fb_mg_create_csr(fb_mg** out, int nl, const fb_csr_host* A, const fb_csr_host* P, const fb_csr_host* R,
                     const uint64_t* const* filter, const uint64_t* fsize, int sigma) {
  if (!out || nl < 1 || nl > kMaxLevels || !A || (nl > 1 && (!P || !R)) || !filter || !fsize) return FB_ERR_INVALID;
  *out = nullptr;
  fb_mg* m = new fb_mg();
  int st = common_init(m);
  if (st != FB_OK) { fb_mg_destroy(m); return st; }
  m->L.resize(nl);
  auto to_host = [](const fb_csr_host& c, HostCsr& h) -> bool {
    if (!c.row_ptr || (c.nnz && (!c.col_ind || !c.val)) || c.row_ptr[c.rows] != c.nnz) return false;
    h.rows = c.rows; h.cols = c.cols;
    h.rp.assign(c.row_ptr, c.row_ptr + c.rows + 1);
    h.ci.resize(c.nnz); h.va.assign(c.val, c.val + c.nnz);
    for (uint64_t k = 0; k < c.nnz; ++k) { if (c.col_ind[k] >= c.cols) return false; h.ci[k] = uint32_t(c.col_ind[k]); }
    return true;
  };
  HostCsr coarseA;
  std::vector<uint32_t> coarseF;
  for (int l = 0; l < nl && st == FB_OK; ++l) {
    HostCsr h;
    if (!to_host(A[l], h) || A[l].rows != A[l].cols || A[l].rows > 0xffffffffull) { st = FB_ERR_INVALID; break; }
    Level& L = m->L[l];
    L.n = uint32_t(A[l].rows);
    std::vector<uint32_t> f(fsize[l]);
    for (uint64_t i = 0; i < fsize[l]; ++i) f[i] = uint32_t(filter[l][i]);
    st = upload_sell(m, L.A, h, sigma < 1 ? 1 : sigma);
    if (st == FB_OK) st = upload_filter(m, L, f);
    if (st == FB_OK && l + 1 < nl) {
      HostCsr hp, hr;
      if (!to_host(P[l], hp) || !to_host(R[l], hr) || P[l].rows != A[l].rows || P[l].cols != A[l + 1].rows ||
          R[l].rows != A[l + 1].rows || R[l].cols != A[l].rows) { st = FB_ERR_INVALID; break; }
      st = upload_csr(m, L.P, hp);
      if (st == FB_OK) st = upload_csr(m, L.R, hr);
    }
    if (l + 1 == nl) { coarseA = std::move(h); coarseF = f; }
  }
  if (st == FB_OK) st = build_coarse_inverse(m, coarseA, coarseF);
  if (st == FB_OK) st = upload_coarse_csr(m, coarseA);
  if (st == FB_OK) st = finish_levels(m);
  if (st != FB_OK) { fb_mg_destroy(m); return st; }
  *out = m;
  return FB_OK;
}

void fb_mg_destroy(fb_mg* m) {
  if (!m) return;
  cudaSetDevice(m->device);
  if (m->stream) cudaStreamSynchronize(m->stream);
  for (int q = 0; q < 2; ++q)
    if (m->g_body[q]) cudaGraphExecDestroy(m->g_body[q]);
  for (void* p : m->allocs) cudaFree(p);
  if (m->host_rr) cudaFreeHost(m->host_rr);
  if (m->ev0) cudaEventDestroy(m->ev0);
  if (m->ev1) cudaEventDestroy(m->ev1);
  if (m->stream) cudaStreamDestroy(m->stream);
  delete m;
}

int fb_mg_solve(fb_mg* m, const double* rhs, double* sol, double* hist, fb_solve_info* info) {
  if (!m || !rhs || !sol) return FB_ERR_INVALID;
  FB_CUDA(cudaSetDevice(m->device));
  return solve_dev(m, rhs, sol, hist, info);
}

static int solve_host(fb_mg* m, const double* rhs_h, double* sol_h, double* hist, fb_solve_info* info, bool zero) {
  if (!m || !rhs_h || !sol_h) return FB_ERR_INVALID;
  if (!m->configured) return FB_ERR_NOT_READY;
  FB_CUDA(cudaSetDevice(m->device));
  FB_TRY(ensure_vectors(m, m->cfg.precision));
  const uint32_t n = m->L[0].n;
  if (!m->hb) { FB_TRY(dalloc(m, &m->hb, n)); FB_TRY(dalloc(m, &m->hx, n)); }
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  FB_CUDA(cudaEventCreate(&e0));
  FB_CUDA(cudaEventCreate(&e1));
  FB_CUDA(cudaEventRecord(e0, m->stream));
  FB_CUDA(cudaMemcpyAsync(m->hb, rhs_h, sizeof(double) * n, cudaMemcpyHostToDevice, m->stream));
  if (zero) FB_CUDA(cudaMemsetAsync(m->hx, 0, sizeof(double) * n, m->stream));
  else FB_CUDA(cudaMemcpyAsync(m->hx, sol_h, sizeof(double) * n, cudaMemcpyHostToDevice, m->stream));
  int st = solve_dev(m, m->hb, m->hx, hist, info);
  if (st == FB_OK) {
    if (cudaMemcpyAsync(sol_h, m->hx, sizeof(double) * n, cudaMemcpyDeviceToHost, m->stream) != cudaSuccess ||
        cudaEventRecord(e1, m->stream) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess) st = FB_ERR_CUDA;
  }
  if (st == FB_OK && info) {
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    info->solve_ms = ms;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return st;
}

int fb_mg_solve_host(fb_mg* m, const double* rhs_h, double* sol_h, double* hist, fb_solve_info* info) {
  return solve_host(m, rhs_h, sol_h, hist, info, false);
}

int fb_mg_solve_host_zero(fb_mg* m, const double* rhs_h, double* sol_h, double* hist, fb_solve_info* info) {
  return solve_host(m, rhs_h, sol_h, hist, info, true);
}

int fb_mg_vcycle(fb_mg* m, const double* def, double* cor) {
  if (!m || !def || !cor) return FB_ERR_INVALID;
  if (!m->configured) return FB_ERR_NOT_READY;
  FB_CUDA(cudaSetDevice(m->device));
  FB_TRY(ensure_vectors(m, m->cfg.precision));
  const uint32_t n = m->L[0].n;
  cudaStream_t s = m->stream;
  if (m->feat_dof) FB_TRY(perm_to_lattice(m, m->r, def, m->feat_dof, n));
  else FB_CUDA(cudaMemcpyAsync(m->r, def, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
  k_dot_rz<double><<<occupancy_grid((const void*)k_dot_rz<double>, n / 32 + 1), 256, 0, s>>>(m->r, m->r, n, m->ws, m->counter, &m->sc->rr);
  FB_CHECK_LAUNCH();
  const void* z = nullptr;
  if (m->cfg.precision != FB_PREC_F64) {
    k_cvt<float, double><<<ew_grid(n), 256, 0, s>>>(m->r32, m->r, n);
    FB_CHECK_LAUNCH();
  }
  FB_TRY(precond(m, &z));
  double* out = cor;
  if (m->feat_dof) {
    if (!m->pv1) FB_TRY(dalloc(m, &m->pv1, n));
    out = m->pv1;
  }
  if (m->cfg.precision == FB_PREC_F64) FB_CUDA(cudaMemcpyAsync(out, z, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
  else { k_cvt<double, float><<<ew_grid(n), 256, 0, s>>>(out, (const float*)z, n); FB_CHECK_LAUNCH(); }
  if (m->feat_dof) FB_TRY(perm_from_lattice(m, cor, out, m->feat_dof, n));
  FB_CUDA(cudaStreamSynchronize(s));
  // a staged kernel whose bounded wait expired left rows unwritten: FB_ERR_TIMEOUT
  return check_kernel_waits(m);
}

int fb_mg_test_expire_wait(fb_mg* m) {
  if (!m || !m->inject) return FB_ERR_INVALID;
  FB_CUDA(cudaSetDevice(m->device));
  const unsigned one = 1u;
  FB_CUDA(cudaMemcpyAsync(m->inject, &one, sizeof(one), cudaMemcpyHostToDevice, m->stream));
  FB_CUDA(cudaStreamSynchronize(m->stream));
  return FB_OK;
}

int fb_mg_time_spmv(fb_mg* m, int level, int which, int prec, int reps, double* ms) {
  if (!m || !ms || level < 0 || level >= (int)m->L.size() || reps < 1 || which < 0 || which > 3 || prec < 0 || prec > 2)
    return FB_ERR_INVALID;
  if (!m->configured) return FB_ERR_NOT_READY;
  FB_CUDA(cudaSetDevice(m->device));
  Level& L = m->L[level];
  const bool low = prec != FB_PREC_F64;
  bool stored;
  if (use_matfree(m, L)) stored = true;
  else if (use_stencil(m, L)) stored = prec == FB_PREC_F64 ? L.St.v64 != nullptr : (prec == FB_PREC_F32 ? L.St.v32 != nullptr : L.St.v16 != nullptr);
  else stored = prec == FB_PREC_F64 ? L.A.v64 != nullptr : (prec == FB_PREC_F32 ? L.A.v32 != nullptr : L.A.v16 != nullptr);
  if ((low && !L.x32) || (!low && !L.x64) || !stored) return FB_ERR_NOT_READY;
  if (which == 2 && (level != 0 || low)) return FB_ERR_INVALID;
  const int saved = m->cfg.precision;
  m->cfg.precision = prec;
  if (which == 3 && (level != 0 || !low || !pcg_p32(m))) {
    m->cfg.precision = saved;
    return FB_ERR_INVALID;
  }
  FB_CUDA(cudaStreamSynchronize(m->stream));
  auto one = [&]() -> int {
    if (!low) {
      double* b = level == 0 ? m->r : L.rhs64;
      if (which == 0) { EpiJacobi<double, false> e{L.x64, b, L.invd64, L.y64, nullptr, L.mask, nullptr, m->cfg.omega_rich}; return spmv_L<double>(m, L, L.x64, e, nullptr); }
      if (which == 1) { EpiDefect<double, false, false> e{L.def64, b, L.mask, nullptr}; return spmv_L<double>(m, L, L.x64, e, nullptr); }
      EpiPcgQ<double> e{m->q, m->p, L.mask};
      return spmv_L<double>(m, L, (const double*)m->p, e, &m->sc->tmp[0]);
    }
    if (which == 3) return pcgq_p32(m, &m->sc->tmp[0], m->p32);
    float* b = level == 0 ? m->r32 : L.rhs32;
    if (which == 0) { EpiJacobi<float, false> e{L.x32, b, L.invd32, L.y32, nullptr, L.mask, nullptr, float(m->cfg.omega_rich)}; return spmv_L<float>(m, L, L.x32, e, nullptr); }
    EpiDefect<float, false, false> e{L.def32, b, L.mask, nullptr};
    return spmv_L<float>(m, L, L.x32, e, nullptr);
  };
  int st = one();  // warm-up
  if (st == FB_OK) st = cuda_status(cudaEventRecord(m->ev0, m->stream));
  for (int i = 0; i < reps && st == FB_OK; ++i) st = one();
  if (st == FB_OK) st = cuda_status(cudaEventRecord(m->ev1, m->stream));
  if (st == FB_OK) st = cuda_status(cudaEventSynchronize(m->ev1));
  if (st == FB_OK) st = check_kernel_waits(m);
  m->cfg.precision = saved;
  if (st != FB_OK) return st;
  float t = 0.0f;
  cudaEventElapsedTime(&t, m->ev0, m->ev1);
  *ms = double(t) / reps;
  return FB_OK;
}

uint64_t fb_mg_num_dofs(const fb_mg* m, int l) {
  if (!m || l < 0 || l >= (int)m->L.size()) return 0;
  return m->L[l].n;
}
int fb_mg_num_levels(const fb_mg* m) { return m ? (int)m->L.size() : 0; }
uint64_t fb_mg_nnz(const fb_mg* m, int l) {
  if (!m || l < 0 || l >= (int)m->L.size()) return 0;
  return m->L[l].A.nnz;
}

}  // extern "C"
