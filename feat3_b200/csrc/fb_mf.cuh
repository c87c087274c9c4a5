// Line-tiled matrix-free Q1 operator for structured 3D levels, staged through shared memory
// by bulk asynchronous copies (cp.async.bulk + mbarrier), with the epilogue of k_mf_q1.
//
// A tile is Lt consecutive interior lattice lines (Y0..Y0+Lt-1, fixed Z) minus their two end
// points, i.e. only rows whose 26 neighbours and 8 cells all exist. Its inputs are contiguous
// ranges: three x ranges (planes Z-1, Z, Z+1; lines Y0-1..Y0+Lt), two k ranges (cell planes
// Z-1, Z; cell lines Y0-1..Y0+Lt-1) and one range per streamed epilogue vector (the tile's
// own lines). One producer warp copies those ranges into an NST-deep ring of stage buffers
// (each range widened to 16-byte boundaries, which the padded allocations of the driver
// allow); eight consumer warps compute TY rows per thread from shared memory, walking up a
// line column with a sliding window (9 new x values and 4 new cell coefficients per row,
// the other 18 + 4 are kept in registers). Rows outside
// the tiles (the lattice boundary planes and lines and the two ends of interior lines) are
// formed by the same warps with direct loads before they take their first tile, while the
// producer's first copies are in flight.
//
// The direct-path rows all lie on the lattice boundary. When the level's filter is exactly that
// boundary (structured hierarchies), every epilogue discards the product of a filtered row
// (Jacobi keeps x, the defect and PCG's q are zero), so the kernel skips their 27-point gathers.
//
// Every wait on an mbarrier is bounded (about one second of %globaltimer); on expiry the
// kernel records the event in `kerr`, stops taking tiles, waits (bounded) for its copies in
// flight and returns, so the host can report the failure with the context intact.
#pragma once
#include "fb_sell.cuh"

#include <type_traits>

namespace fb {

// ------------------------------------------------------------------ staged epilogues
// Epilogues whose row-streamed inputs the tiled kernel stages in shared memory. `apply`
// receives the product s, the row's own x value xc and the staged stream values st[].
template<typename Epi> struct Staged { static constexpr bool kOk = false; static constexpr int kStreams = 0; };

template<typename T, bool RED, bool DOT>
struct Staged<EpiJacobi<T, RED, DOT>> {
  using E = EpiJacobi<T, RED, DOT>;
  static constexpr bool kOk = true;
  static constexpr int kStreams = 2;
  static const void* stream(const E& e, int i) { return i == 0 ? (const void*)e.rhs : (const void*)e.invd; }
  static bool input_is_x(const E& e, const void* x) { return e.x == x; }
  static const uint32_t* mask(const E& e) { return e.mask; }
  __device__ static bool skip(const E& e) { return smoother_skip<T>(e.skip_src); }
  __device__ __forceinline__ static double apply(const E& e, bool skp, uint32_t row, T s, T xc, const T* st, bool m,
                                                 T) {
    if (skp) {
      const T o = e.s0 ? e.s0[row] : T(0);
      e.out[row] = o;
      return DOT ? double(o) * double(st[0]) : 0.0;
    }
    const T d = st[0] - s;
    if (m) {
      e.out[row] = xc;
      return DOT ? double(xc) * double(st[0]) : 0.0;
    }
    const T t = st[1] * d;
    const T o = e.omega * t + xc;
    e.out[row] = o;
    return RED ? double(d) * double(d) : (DOT ? double(o) * double(st[0]) : 0.0);
  }
};

template<typename T, bool RED, bool DOT>
struct Staged<EpiJacobiK<T, RED, DOT>> {
  using E = EpiJacobiK<T, RED, DOT>;
  static constexpr bool kOk = true;
  static constexpr int kStreams = 1;
  static const void* stream(const E& e, int) { return e.rhs; }
  static bool input_is_x(const E& e, const void* x) { return e.x == x; }
  static const uint32_t* mask(const E& e) { return e.mask; }
  __device__ static bool skip(const E& e) { return smoother_skip<T>(e.skip_src); }
  __device__ __forceinline__ static double apply(const E& e, bool skp, uint32_t row, T s, T xc, const T* st, bool m,
                                                 T kc) {
    if (skp) {
      const T o = e.s0 ? e.s0[row] : T(0);
      e.out[row] = o;
      return DOT ? double(o) * double(st[0]) : 0.0;
    }
    const T d = st[0] - s;
    if (m) {
      e.out[row] = xc;
      return DOT ? double(xc) * double(st[0]) : 0.0;
    }
    const T t = __fdividef(e.wd, kc) * d;
    const T o = e.omega * t + xc;
    e.out[row] = o;
    return RED ? double(d) * double(d) : (DOT ? double(o) * double(st[0]) : 0.0);
  }
};

template<typename T, bool RED, bool LOW>
struct Staged<EpiDefect<T, RED, LOW>> {
  using E = EpiDefect<T, RED, LOW>;
  static constexpr bool kOk = true;
  static constexpr int kStreams = 1;
  static const void* stream(const E& e, int) { return e.rhs; }
  static bool input_is_x(const E&, const void*) { return true; }
  static const uint32_t* mask(const E& e) { return e.mask; }
  __device__ static bool skip(const E&) { return false; }
  __device__ __forceinline__ static double apply(const E& e, bool, uint32_t row, T s, T, const T* st, bool m, T) {
    T d = st[0] - s;
    if (m) d = T(0);
    e.def[row] = d;
    if (LOW) e.def32[row] = float(d);
    return RED ? double(d) * double(d) : 0.0;
  }
};

template<typename T, typename PT>
struct Staged<EpiPcgQ<T, PT>> {
  using E = EpiPcgQ<T, PT>;
  static constexpr bool kOk = true;
  static constexpr int kStreams = 0;
  static const void* stream(const E&, int) { return nullptr; }
  static bool input_is_x(const E& e, const void* x) { return e.p == x; }  // q . p with p the product's input
  static const uint32_t* mask(const E& e) { return e.mask; }
  __device__ static bool skip(const E&) { return false; }
  __device__ __forceinline__ static double apply(const E& e, bool, uint32_t row, T s, T xc, const T*, bool m, T) {
    const T v = m ? T(0) : s;
    e.q[row] = v;
    return double(v) * double(xc);
  }
};

// ------------------------------------------------------------------ tile geometry
// A tile holds Lt = G * TY consecutive interior lines of one interior plane: G groups of W
// threads (W = M1 - 2, one thread per interior point of a line), each group walking TY
// consecutive lines with a sliding register window.
struct MfTile {
  uint32_t M1, N;        // lattice points and cells per side
  uint32_t G, Lt, tpp;   // thread groups, lines per tile (G * TY), tiles per interior plane
  uint32_t ntiles;       // (M1 - 2) * tpp
  uint32_t cap_x, cap_k, cap_s, cap_m;  // bytes reserved per x / k / stream / mask range in a stage
  uint32_t stage_bytes;
  uint32_t nbl_items;    // direct-path items: boundary-line chunks
  uint32_t nedge_items;  // direct-path items: 16 interior lines' end points each
  uint32_t dz, dyt;      // grid stride in tiles, as (planes, tiles within a plane) = divmod(gridDim, tpp)
  uint32_t direct_masked;  // the filter is the lattice boundary: every direct-path row is filtered, and
                           // the epilogue of a filtered row does not read the product
  unsigned* inject;        // test hook (fb_mg_test_expire_wait), or null: while *inject is set, block 0's
                           // producer clears it and leaves its first stage unfilled (no copy, no arrive)
};

// tiles of a block in grid-stride order without divisions in the loop
struct TileIter {
  uint32_t Z, yt;  // plane (1-based interior plane index) and tile within the plane
  __device__ __forceinline__ TileIter(const MfTile& G, uint32_t t0) : Z(1 + t0 / G.tpp), yt(t0 % G.tpp) {}
  __device__ __forceinline__ void next(const MfTile& G) {
    yt += G.dyt;
    Z += G.dz;
    if (yt >= G.tpp) { yt -= G.tpp; ++Z; }
  }
};
struct TileGeo {
  uint32_t Z, Y0, lt;
};
__device__ __forceinline__ TileGeo tile_geo(const MfTile& G, const TileIter& ti) {
  TileGeo g;
  g.Z = ti.Z;
  g.Y0 = 1 + ti.yt * G.Lt;
  const uint32_t rem = G.M1 - 1 - g.Y0;  // interior lines left in the plane
  g.lt = rem < G.Lt ? rem : G.Lt;
  return g;
}

// ------------------------------------------------------------------ mbarrier / bulk copy
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* b, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive_tx(uint64_t* b, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.release.cta.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(b)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* b) {
  asm volatile("mbarrier.arrive.release.cta.shared::cta.b64 _, [%0];" ::"r"(smem_u32(b)) : "memory");
}
__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
// wait for the phase of parity `ph` to complete; false after ~1 s
__device__ __forceinline__ bool mbar_wait(uint64_t* b, uint32_t ph) {
  const uint32_t a = smem_u32(b);
  uint32_t done = 0;
  uint64_t t0 = 0;
  for (uint32_t it = 0;; ++it) {
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.acquire.cta.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(a), "r"(ph)
        : "memory");
    if (done) return true;
    if (it == 0) t0 = global_ns();
    else if ((it & 63) == 0 && global_ns() - t0 > 1000000000ull) return false;
  }
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

// range [lo, hi] (elements) of `base` widened to 16-byte boundaries: start element, bytes
template<typename T>
__device__ __forceinline__ void widen(uint64_t lo, uint64_t hi, uint64_t& alo, uint32_t& bytes) {
  constexpr uint64_t E = 16 / sizeof(T);
  alo = lo & ~(E - 1);
  bytes = uint32_t(((hi + 1 - alo) * sizeof(T) + 15) & ~uint64_t(15));
}

// ------------------------------------------------------------------ direct-path row
// A(k) x for one row at lattice point (X, Y, Z) with clamped gathers (any row of the level)
template<typename T, typename XT = T>
__device__ __forceinline__ T mf_row_direct(const MfView<T, 3>& A, const XT* __restrict__ x, int32_t row, int32_t X,
                                           int32_t Y, int32_t Z) {
  const int32_t last = int32_t(A.rows) - 1;
  const int32_t N = int32_t(A.M1) - 1;
  T xv[27];
#pragma unroll
  for (int j = 0; j < 27; ++j) {
    int32_t col = row + A.off[j];
    col = col < 0 ? 0 : (col > last ? last : col);
    xv[j] = T(__ldg(x + col));
  }
  T s = T(0);
#pragma unroll
  for (int e = 0; e < 8; ++e) {
    const int ox = e & 1, oy = (e >> 1) & 1, oz = (e >> 2) & 1;
    const int a = (1 - ox) | ((1 - oy) << 1) | ((1 - oz) << 2);
    const int32_t ex = X - 1 + ox, ey = Y - 1 + oy, ez = Z - 1 + oz;
    const bool valid = uint32_t(ex) < uint32_t(N) && uint32_t(ey) < uint32_t(N) && uint32_t(ez) < uint32_t(N);
    const int64_t eidx = valid ? int64_t(ex) + int64_t(N) * (ey + int64_t(N) * ez) : 0;
    T ke = A.k ? __ldg(A.k + eidx) : T(1);
    ke = valid ? ke : T(0);
    T in = T(0);
#pragma unroll
    for (int b = 0; b < 8; ++b) {
      const int dx = ox - 1 + (b & 1), dy = oy - 1 + ((b >> 1) & 1), dz = oz - 1 + ((b >> 2) & 1);
      in += A.kr[a ^ b] * xv[(dz + 1) * 9 + (dy + 1) * 3 + (dx + 1)];
    }
    s += ke * in;
  }
  return s;
}

// ------------------------------------------------------------------ rows outside the tiles
// The lattice boundary lines in items of 32 consecutive rows ((M1 + 31) / 32 items per line:
// planes Z = 0 and M1-1 first, then lines Y = 0 and M1-1 of every interior plane), then the two
// end points of every interior line in items of 16 lines. Item -> this lane's row (-1: none) and
// its lattice point.
__device__ __forceinline__ int32_t direct_row(uint32_t item, uint32_t lane, uint32_t M1, uint32_t nbl_items,
                                              uint32_t& X, uint32_t& Y, uint32_t& Z) {
  const uint32_t W = M1 - 2, cpl = (M1 + 31) / 32;
  if (item < nbl_items) {
    const uint32_t bl = item / cpl;
    X = (item - bl * cpl) * 32 + lane;
    if (bl < 2 * M1) {
      Z = bl < M1 ? 0 : M1 - 1;
      Y = bl < M1 ? bl : bl - M1;
    } else {
      const uint32_t r = bl - 2 * M1;
      Z = 1 + (r >> 1);
      Y = (r & 1) ? M1 - 1 : 0;
    }
    return X < M1 ? int32_t((Z * M1 + Y) * M1 + X) : -1;
  }
  const uint32_t li = (item - nbl_items) * 16 + (lane >> 1);
  if (li >= W * W) return -1;
  const uint32_t zq = li / W;
  Y = 1 + (li - zq * W);
  Z = 1 + zq;
  X = (lane & 1) ? M1 - 1 : 0;
  return int32_t((Z * M1 + Y) * M1 + X);
}

// One warp's share of the rows outside the tiles (items first, first + stride, ...), epilogue
// applied; returns the thread's reduction terms in item order. When the epilogue's filter is the
// lattice boundary (`masked`), every such row is filtered: the product is not formed, and the x
// and first streamed values of four items (two in FP64) are loaded before any is used, so that a
// warp's items wait for memory once per four rather than once each. Otherwise A(k) x is formed by
// gathers.
template<typename T, typename XT, typename Epi>
__device__ __forceinline__ double direct_rows(const MfView<T, 3>& A, const XT* __restrict__ x, const Epi& epi,
                                              const T* st0, bool skp, uint32_t M1, uint32_t nbl_items,
                                              uint32_t nitems, bool masked, uint32_t first, uint32_t stride,
                                              uint32_t lane) {
  using SE = Staged<Epi>;
  double acc = 0.0;
  uint32_t X = 0, Y = 0, Z = 0;
  if (masked) {
    constexpr int B = sizeof(T) == 4 ? 4 : 2;
    for (uint32_t i0 = first; i0 < nitems; i0 += B * stride) {
      int32_t rows[B];
      T xv[B], sv[B];
#pragma unroll
      for (int b = 0; b < B; ++b) {
        const uint32_t item = i0 + uint32_t(b) * stride;
        rows[b] = item < nitems ? direct_row(item, lane, M1, nbl_items, X, Y, Z) : -1;
      }
#pragma unroll
      for (int b = 0; b < B; ++b) {
        xv[b] = rows[b] >= 0 ? T(x[rows[b]]) : T(0);
        sv[b] = (SE::kStreams > 0 && rows[b] >= 0) ? st0[rows[b]] : T(0);
      }
#pragma unroll
      for (int b = 0; b < B; ++b)
        if (rows[b] >= 0) acc += SE::apply(epi, skp, uint32_t(rows[b]), T(0), xv[b], &sv[b], true, T(0));
    }
    return acc;
  }
  for (uint32_t item = first; item < nitems; item += stride) {
    const int32_t row = direct_row(item, lane, M1, nbl_items, X, Y, Z);
    if (row >= 0) acc += epi(uint32_t(row), mf_row_direct<T, XT>(A, x, row, int32_t(X), int32_t(Y), int32_t(Z)));
  }
  return acc;
}

// sums of the cell coefficients of cell line c (kw[oz][c][ox]) over the cells that a
// neighbour offset (dz, dx) in {-1,0,1}^2 selects: -1 -> the lower cell, +1 -> the upper one,
// 0 -> both; K[dz+1][dx+1]
template<typename T>
__device__ __forceinline__ void ksums(const T (&kw)[2][2][2], int c, T (&K)[3][3]) {
  const T k00 = kw[0][c][0], k01 = kw[0][c][1], k10 = kw[1][c][0], k11 = kw[1][c][1];
  K[0][0] = k00; K[0][2] = k01; K[2][0] = k10; K[2][2] = k11;
  K[0][1] = k00 + k01; K[2][1] = k10 + k11;
  K[1][0] = k00 + k10; K[1][2] = k01 + k11;
  K[1][1] = K[0][1] + K[2][1];
}

// the same sums with the two cell planes packed: kp[ex] = (k of plane Z-1, k of plane Z) for
// cell columns ex = 0, 1 of one cell line; Kp[dx] = (K[0][dx], K[2][dx]), Km[dx] = K[1][dx]
__device__ __forceinline__ void ksums2(const float2 (&kp)[2], float2 (&Kp)[3], float (&Km)[3]) {
  Kp[0] = kp[0];
  Kp[2] = kp[1];
  Kp[1] = __fadd2_rn(kp[0], kp[1]);
  Km[0] = kp[0].x + kp[0].y;
  Km[2] = kp[1].x + kp[1].y;
  Km[1] = Kp[1].x + Kp[1].y;
}

// ------------------------------------------------------------------ the tiled kernel
// 8 consumer warps + 1 producer warp; dynamic shared memory = NST * G.stage_bytes.
// CM1: the lattice size as a compile-time constant (0: G.M1 at run time), which turns the
// shared-memory offsets of the window walk into immediates on the levels that dominate.
// XT: storage type of the input vector x (FP32 for an FP64 product of an FP32-stored vector);
// the window and the arithmetic are in T.
template<typename T, typename Epi, int NST, int MINB, int TY, int CM1, typename XT = T>
__global__ void __launch_bounds__(288, MINB) k_mf_q1_tiled(MfView<T, 3> A, MfTile G, const XT* __restrict__ x, Epi epi,
                                                           const T* st0, const T* st1, const uint32_t* mask,
                                                           double* ws, unsigned* counter, double* red_out,
                                                           unsigned* kerr) {
  using SE = Staged<Epi>;
  constexpr int NS = SE::kStreams;
  constexpr uint64_t E = 16 / sizeof(T);
  constexpr uint64_t EX = 16 / sizeof(XT);
  // FP32 throughout: the stencil runs on packed FP32 pairs (fma.rn.f32x2)
  constexpr bool PK = std::is_same<T, float>::value && std::is_same<XT, float>::value;
  pdl_wait();
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ uint64_t full[NST], empty[NST];
  __shared__ double sh[16];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < NST; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 8);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  const uint32_t M1 = CM1 ? uint32_t(CM1) : G.M1, N = M1 - 1;
  const uint32_t W = M1 - 2;  // interior points per line
  // stage layout: x planes | k cell planes | streams | mask words
  const uint32_t off_k = 3 * G.cap_x, off_s = off_k + 2 * G.cap_k, off_m = off_s + NS * G.cap_s;
  double acc = 0.0;
  if (warp == 8) {
    // ---------------- producer: lane q computes and issues copy q of the tile
    // (0-2: x planes, 3-4: cell planes, 5-6: streams, 7: mask words)
    uint32_t it = 0;
    bool stop = false;
    TileIter ti(G, blockIdx.x);
    for (uint32_t t = blockIdx.x; t < G.ntiles; t += gridDim.x, ++it, ti.next(G)) {
      const int s = int(it % NST);
      const uint32_t ph = (it / NST) & 1u;
      if (G.inject && it == 0 && blockIdx.x == 0) {
        // test hook: nothing arrives on this stage, so the consumers' bounded wait on it expires
        // (then the producer's wait on its release, then the drain's); no copy is issued for it
        unsigned v = 0;
        if (lane == 0 && *reinterpret_cast<volatile unsigned*>(G.inject)) v = atomicExch(G.inject, 0u);
        if (__shfl_sync(0xffffffffu, v, 0)) continue;
      }
      if (it >= NST) {
        const bool okw = lane == 0 ? mbar_wait(&empty[s], ph ^ 1u) : true;
        if (!__shfl_sync(0xffffffffu, okw, 0)) {
          if (lane == 0) atomicExch(kerr, 1u);
          stop = true;
          break;
        }
      }
      const TileGeo g = tile_geo(G, ti);
      unsigned char* st = smem + size_t(s) * G.stage_bytes;
      const uint64_t r0 = (uint64_t(g.Z) * M1 + g.Y0) * M1, r1 = r0 + uint64_t(g.lt) * M1 - 1;
      uint64_t lo = 0;
      uint32_t by = 0, dst = 0;
      const void* src = nullptr;
      if (lane < 3) {
        const uint64_t zp = g.Z - 1 + lane;
        widen<XT>((zp * M1 + g.Y0 - 1) * M1, (zp * M1 + g.Y0 + g.lt) * M1 + M1 - 1, lo, by);
        src = x + lo;
        dst = lane * G.cap_x;
      } else if (lane < 5) {
        if (A.k) {
          const uint64_t ez = g.Z - 1 + (lane - 3);
          widen<T>((ez * N + g.Y0 - 1) * N, (ez * N + g.Y0 + g.lt - 1) * N + N - 1, lo, by);
          src = A.k + lo;
          dst = off_k + (lane - 3) * G.cap_k;
        }
      } else if (lane < 7) {
        if (lane - 5 < NS) {
          widen<T>(r0, r1, lo, by);
          src = (lane == 5 ? st0 : st1) + lo;
          dst = off_s + (lane - 5) * G.cap_s;
        }
      } else if (lane == 7) {
        if (mask) {
          widen<uint32_t>(r0 >> 5, r1 >> 5, lo, by);
          src = mask + lo;
          dst = off_m;
        }
      }
      uint32_t total = by;
#pragma unroll
      for (int o = 4; o > 0; o >>= 1) total += __shfl_xor_sync(0xffffffffu, total, o);
      if (lane == 0) mbar_arrive_tx(&full[s], total);
      __syncwarp();
      if (by) bulk_g2s(st + dst, src, by, &full[s]);
    }
    // copies still in flight (none unless the consumers stopped early)
    (void)stop;
    if (lane == 0) {
      const uint32_t issued = it;
      for (uint32_t j = issued > NST ? issued - NST : 0; j < issued; ++j)
        if (!mbar_wait(&full[j % NST], (j / NST) & 1u)) atomicExch(kerr, 2u);
    }
    __syncwarp();
  } else {
    // ---------------- direct path first: the rows no tile holds, while the producer fills the
    // first stages
    const bool skp = SE::skip(epi);
    acc += direct_rows<T, XT, Epi>(A, x, epi, st0, skp, M1, G.nbl_items, G.nbl_items + G.nedge_items,
                                   G.direct_masked != 0, blockIdx.x * 8 + warp, gridDim.x * 8, lane);
    // ---------------- consumers: TY rows per thread and tile (sliding window along Y)
    const uint32_t tid = threadIdx.x;
    const uint32_t grp = tid / W, X = 1 + (tid - grp * W);
    const bool active = grp < G.G;
    uint32_t it = 0;
    TileIter ti(G, blockIdx.x);
    for (uint32_t t = blockIdx.x; t < G.ntiles; t += gridDim.x, ++it, ti.next(G)) {
      const int s = int(it % NST);
      const uint32_t ph = (it / NST) & 1u;
      if (!mbar_wait(&full[s], ph)) {
        atomicExch(kerr, 3u);
        break;
      }
      const TileGeo g = tile_geo(G, ti);
      const unsigned char* st = smem + size_t(s) * G.stage_bytes;
      const uint32_t l0 = grp * TY;  // first line of this group, relative to Y0
      if (active && l0 < g.lt) {
        // window origin: x line Y0-1+l0 of each plane, k cell line Y0-1+l0, at this X
        const XT* xs[3];
#pragma unroll
        for (int q = 0; q < 3; ++q) {
          const uint64_t zp = g.Z - 1 + q;
          const uint64_t xlo = (zp * M1 + g.Y0 - 1) * M1;
          xs[q] = reinterpret_cast<const XT*>(st + q * G.cap_x) + (xlo & (EX - 1)) + l0 * M1 + X;
        }
        const T* ks[2] = {nullptr, nullptr};
        if (A.k) {
#pragma unroll
          for (int q = 0; q < 2; ++q) {
            const uint64_t ez = g.Z - 1 + q;
            const uint64_t klo = (ez * N + g.Y0 - 1) * N;
            ks[q] = reinterpret_cast<const T*>(st + off_k + q * G.cap_k) + (klo & (E - 1)) + l0 * N + (X - 1);
          }
        }
        const uint32_t r0 = (g.Z * M1 + g.Y0) * M1;  // rows < 2^31 (checked by the launcher)
        const T* ss = reinterpret_cast<const T*>(st + off_s) + (r0 & uint32_t(E - 1)) + l0 * M1 + X;
        const uint32_t* ms = reinterpret_cast<const uint32_t*>(st + off_m);
        const uint32_t mw0 = (r0 >> 5) & ~3u;  // first staged mask word
        // window: xw[plane][line][dx], kw[cell plane][cell line][ex]; in the packed FP32 form
        // xp[line][dx] pairs planes Z-1 and Z+1, xm[line][dx] is plane Z, kp[cell line][ex]
        // pairs cell planes Z-1 and Z (the unused form's arrays are dead code)
        T xw[3][3][3], kw[2][2][2];
        float2 xp[3][3], kp[2][2], Kp[2][3];
        T xm[3][3], Km[2][3];
        // per cell line: sums of k over the cells selected by (dz, dx) in {-1,0,1}^2
        T K[2][3][3];
        if constexpr (PK) {
#pragma unroll
          for (int l = 0; l < 2; ++l)
#pragma unroll
            for (int d = 0; d < 3; ++d) {
              xp[l][d] = make_float2(xs[0][l * int(M1) + d - 1], xs[2][l * int(M1) + d - 1]);
              xm[l][d] = xs[1][l * int(M1) + d - 1];
            }
#pragma unroll
          for (int c = 0; c < 2; ++c) kp[0][c] = A.k ? make_float2(ks[0][c], ks[1][c]) : make_float2(1.f, 1.f);
          ksums2(kp[0], Kp[0], Km[0]);
        } else {
#pragma unroll
          for (int q = 0; q < 3; ++q)
#pragma unroll
            for (int l = 0; l < 2; ++l)
#pragma unroll
              for (int d = 0; d < 3; ++d) xw[q][l][d] = T(xs[q][l * int(M1) + d - 1]);
#pragma unroll
          for (int q = 0; q < 2; ++q) {
            kw[q][0][0] = A.k ? ks[q][0] : T(1);
            kw[q][0][1] = A.k ? ks[q][1] : T(1);
          }
          ksums(kw, 0, K[0]);
        }
        // FAST: every line of the group lies in the tile, the coefficients are given, no filter
        // word is staged and the smoother runs: rows without a branch, so the loads of a row
        // can be scheduled ahead of the previous row's epilogue
        auto rows = [&](auto fast) {
          constexpr bool FAST = decltype(fast)::value;
#pragma unroll
          for (int j = 0; j < TY; ++j) {
            if (!FAST && l0 + j >= g.lt) break;
            T s, kc, xc;
            if constexpr (PK) {
              // packed FP32 form: the neighbours in planes Z-1 and Z+1 pair up (same line and
              // column, lanes x and y), two FP32 operations per instruction; the terms are those
              // of the scalar form, summed plane pair by plane pair
#pragma unroll
              for (int d = 0; d < 3; ++d) {
                xp[2][d] = make_float2(xs[0][(j + 2) * int(M1) + d - 1], xs[2][(j + 2) * int(M1) + d - 1]);
                xm[2][d] = xs[1][(j + 2) * int(M1) + d - 1];
              }
#pragma unroll
              for (int c = 0; c < 2; ++c)
                kp[1][c] = (FAST || A.k) ? make_float2(ks[0][(j + 1) * N + c], ks[1][(j + 1) * N + c])
                                         : make_float2(1.f, 1.f);
              ksums2(kp[1], Kp[1], Km[1]);
              kc = Km[0][1] + Km[1][1];  // the row's 8 cells
              // r = 5 (dx != 1, dy = 1), 6 (dx = 1, dy != 1), 7 (dx, dy != 1), planes Z-1 / Z+1
              float2 S5 = __fmul2_rn(__fadd2_rn(Kp[0][0], Kp[1][0]), xp[1][0]);
              S5 = __ffma2_rn(__fadd2_rn(Kp[0][2], Kp[1][2]), xp[1][2], S5);
              float2 S6 = __fmul2_rn(Kp[0][1], xp[0][1]);
              S6 = __ffma2_rn(Kp[1][1], xp[2][1], S6);
              float2 S7 = __fmul2_rn(Kp[0][0], xp[0][0]);
              S7 = __ffma2_rn(Kp[0][2], xp[0][2], S7);
              S7 = __ffma2_rn(Kp[1][0], xp[2][0], S7);
              S7 = __ffma2_rn(Kp[1][2], xp[2][2], S7);
              // plane Z: the centre (r = 0) and r = 3 (dx, dy != 1)
              const T S0 = kc * xm[1][1];
              T S3 = Km[0][0] * xm[0][0];
              S3 += Km[0][2] * xm[0][2];
              S3 += Km[1][0] * xm[2][0];
              S3 += Km[1][2] * xm[2][2];
              s = A.kr[0] * S0;
              s += A.kr[3] * S3;
              s += A.kr[5] * (S5.x + S5.y);
              s += A.kr[6] * (S6.x + S6.y);
              s += A.kr[7] * (S7.x + S7.y);
              xc = xm[1][1];
            } else {
#pragma unroll
              for (int q = 0; q < 3; ++q)
#pragma unroll
                for (int d = 0; d < 3; ++d) xw[q][2][d] = T(xs[q][(j + 2) * int(M1) + d - 1]);
              if (FAST || A.k) {
#pragma unroll
                for (int q = 0; q < 2; ++q) {
                  kw[q][1][0] = ks[q][(j + 1) * N];
                  kw[q][1][1] = ks[q][(j + 1) * N + 1];
                }
              } else {
#pragma unroll
                for (int q = 0; q < 2; ++q) kw[q][1][0] = kw[q][1][1] = T(1);
              }
              // stencil form of the cell sum: the coefficient of neighbour d is kr[r(d)] times the
              // sum of k over the cells holding both the row's node and d, where r(d) has a bit for
              // every direction in which d is nonzero (K_ref[a][b] = kr[a ^ b]). The 6 face
              // neighbours (one bit in r) have coefficient 0 for the Q1 Laplacian of a cube (the
              // launcher checks kr[1], kr[2], kr[4] are of rounding size) and are left out.
              ksums(kw, 1, K[1]);
              kc = K[0][1][1] + K[1][1][1];  // the row's 8 cells
              T S[8];
#pragma unroll
              for (int r = 0; r < 8; ++r) S[r] = T(0);
#pragma unroll
              for (int dz = 0; dz < 3; ++dz)
#pragma unroll
                for (int dy = 0; dy < 3; ++dy)
#pragma unroll
                  for (int dx = 0; dx < 3; ++dx) {
                    const int r = (dx != 1 ? 1 : 0) | (dy != 1 ? 2 : 0) | (dz != 1 ? 4 : 0);
                    if (r == 1 || r == 2 || r == 4) continue;
                    const T Kd = dy == 0 ? K[0][dz][dx] : (dy == 2 ? K[1][dz][dx] : K[0][dz][dx] + K[1][dz][dx]);
                    S[r] += Kd * xw[dz][dy][dx];
                  }
              s = A.kr[0] * S[0];
#pragma unroll
              for (int r = 3; r < 8; ++r)
                if (r != 4) s += A.kr[r] * S[r];
              xc = xw[1][1][1];
            }
            const uint32_t row = r0 + (l0 + j) * M1 + X;
            T sv[NS > 0 ? NS : 1];
            if (NS > 0) sv[0] = ss[j * int(M1)];
            if (NS > 1)
              sv[NS > 1 ? 1 : 0] =
                  reinterpret_cast<const T*>(reinterpret_cast<const unsigned char*>(ss) + G.cap_s)[j * int(M1)];
            const bool mb = (!FAST && mask) ? ((ms[(row >> 5) - mw0] >> (row & 31)) & 1u) : false;
            acc += SE::apply(epi, FAST ? false : skp, row, s, xc, sv, mb, kc);
            // slide the window one line up
            if constexpr (PK) {
#pragma unroll
              for (int d = 0; d < 3; ++d) {
                xp[0][d] = xp[1][d];
                xp[1][d] = xp[2][d];
                xm[0][d] = xm[1][d];
                xm[1][d] = xm[2][d];
                Kp[0][d] = Kp[1][d];
                Km[0][d] = Km[1][d];
              }
              kp[0][0] = kp[1][0];
              kp[0][1] = kp[1][1];
            } else {
#pragma unroll
              for (int q = 0; q < 3; ++q)
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                  xw[q][0][d] = xw[q][1][d];
                  xw[q][1][d] = xw[q][2][d];
                }
#pragma unroll
              for (int q = 0; q < 2; ++q) {
                kw[q][0][0] = kw[q][1][0];
                kw[q][0][1] = kw[q][1][1];
              }
#pragma unroll
              for (int a = 0; a < 3; ++a)
#pragma unroll
                for (int b = 0; b < 3; ++b) K[0][a][b] = K[1][a][b];
            }
          }
        };
        if (!skp && !mask && A.k && l0 + TY <= g.lt) rows(std::true_type{});
        else rows(std::false_type{});
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(&empty[s]);
    }
  }
  pdl_trigger();
  if (Epi::kReduce) {
    const double blk = block_sum<288>(acc, sh);
    reduce_finish<288>(blk, ws, counter, red_out, sh, false);
  }
}

}  // namespace fb
