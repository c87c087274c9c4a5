// Streaming form of the matrix-free Q1 operator on the two finest structured 3D levels
// (lattice size a compile-time constant), with the epilogues of k_mf_q1_tiled.
//
// The interior planes form slabs of G consecutive planes, one thread group per plane and one thread
// per interior point X of a line (or per two, CPT = 2). The slab-lines (slab, interior line Y)
// are numbered u = slab * W + (Y - 1), and each CTA takes one contiguous range of them, walking up
// the lines of a slab with a sliding 3x3x3 register window that it carries from stage to stage:
// a run starts with an init stage (x lines Y-1 and Y, cell line Y-1, no rows), and then every
// stage brings only the lines its TY rows need for the first time (x line Y+1 and cell line Y of
// each row Y, plus the streamed epilogue inputs). No line is loaded twice within a run, and the
// stages are small, so several (NST) are in flight per CTA.
//
// The window's line slots are named modulo 3 (x) and modulo 2 (cell lines) by the row's position
// in its stage; every stage of a run but its last has exactly TY rows (a multiple of 6), so the
// names repeat from stage to stage and the window never moves between registers.
//
// One producer warp issues the stage's bulk copies (cp.async.bulk + mbarrier, each range widened
// to 16-byte boundaries, which the padded allocations allow); NCW (8, 12 or 16) consumer warps compute. Rows
// outside the slabs' interiors (the lattice boundary) are formed first by the consumer warps with
// direct loads, as in k_mf_q1_tiled. Every mbarrier wait is bounded (about one second); on expiry
// the kernel records it in `kerr`, stops, waits (bounded) for its own copies and returns.
#pragma once
#include "fb_mf.cuh"

namespace fb {

struct MfStream {
  uint32_t G;                      // planes per slab (thread groups of W threads)
  uint32_t nslab;                  // ceil(W / G)
  uint64_t units;                  // nslab * W slab-lines
  uint32_t cap_x, cap_k, cap_s;    // bytes reserved per x / cell / stream range in a stage
  uint32_t stage_bytes;
  uint32_t nbl_items, nedge_items; // direct-path items, as MfTile
  uint32_t direct_masked;          // as MfTile
  unsigned* inject;                // test hook, as MfTile
};

// one stage of a CTA's run: TY (or fewer, at the end of a slab or of the range) rows starting at
// interior line y of a slab, or the init stage of a run (x lines y-1, y and cell line y-1)
struct StreamStep {
  uint32_t slab, y, nl;
  bool init;
};

template<uint32_t W, int TY>
struct StreamIter {
  uint64_t cur, end;
  uint32_t last_slab = 0xffffffffu;
  __device__ __forceinline__ StreamIter(uint64_t u0, uint64_t u1) : cur(u0), end(u1) {}
  __device__ __forceinline__ bool next(StreamStep& st) {
    if (cur >= end) return false;
    const uint32_t slab = uint32_t(cur / W), y = uint32_t(cur - uint64_t(slab) * W) + 1;
    if (slab != last_slab) {
      last_slab = slab;
      st = {slab, y, 0u, true};
      return true;
    }
    uint64_t nl = uint64_t(TY);
    nl = nl < uint64_t(W + 1 - y) ? nl : uint64_t(W + 1 - y);
    nl = nl < end - cur ? nl : end - cur;
    st = {slab, y, uint32_t(nl), false};
    cur += nl;
    return true;
  }
};

// NCW consumer warps (8, 12 or 16) and one producer warp per CTA. CPT = 2: each consumer thread forms
// two adjacent rows X0 = 1 + 2t and X0 + 1 of a line from one window of 4 columns and 3 cells
// (packed FP32 form only); the last thread of an odd-width line computes its second row on the
// lattice boundary from in-slot data and does not store it.
template<typename T, typename Epi, int NST, int TY, int CM1, typename XT, int NCW, int CPT>
__device__ __forceinline__ void mf_stream_body(const MfView<T, 3>& A, const MfStream& G, const XT* __restrict__ x,
                                               const Epi& epi, const T* st0, const T* st1, double* ws,
                                               unsigned* counter, double* red_out, unsigned* kerr) {
  static_assert(TY % 6 == 0, "window slots repeat every 6 rows");
  static_assert(CPT == 1 || (CPT == 2 && std::is_same<T, float>::value && std::is_same<XT, float>::value &&
                             Staged<Epi>::kStreams <= 1),
                "two rows per thread: packed FP32 form, at most one streamed vector");
  constexpr int NT = 32 * (NCW + 1);
  using SE = Staged<Epi>;
  constexpr int NS = SE::kStreams;
  constexpr uint32_t M1 = CM1, N = M1 - 1, W = M1 - 2;
  constexpr uint64_t E = 16 / sizeof(T);
  constexpr uint64_t EX = 16 / sizeof(XT);
  constexpr bool PK = std::is_same<T, float>::value && std::is_same<XT, float>::value;
  pdl_wait();
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ uint64_t full[NST], empty[NST];
  __shared__ double sh[NT / 32];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < NST; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], NCW);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  const uint32_t Gp = G.G;
  // stage layout: (G+2) x planes | (G+1) cell planes | NS * G stream planes
  const uint32_t off_k = (Gp + 2) * G.cap_x, off_s = off_k + (Gp + 1) * G.cap_k;
  const uint64_t u0 = G.units * blockIdx.x / gridDim.x, u1 = G.units * (blockIdx.x + 1) / gridDim.x;
  double acc = 0.0;
  if (warp == NCW) {
    // ---------------- producer: lane q issues range q of the stage
    // (0..G+1: x planes Z0-1..Z0+G; G+2..2G+2: cell planes Z0-1..Z0+G-1; then the streams)
    uint32_t it = 0;
    StreamIter<W, TY> sit(u0, u1);
    StreamStep stp;
    while (sit.next(stp)) {
      const int s = int(it % NST);
      const uint32_t ph = (it / NST) & 1u;
      if (G.inject && it == 0 && blockIdx.x == 0) {
        // test hook: nothing arrives on this stage, so the consumers' bounded wait on it expires
        // (then the producer's wait on its release, then the drain's); no copy is issued for it
        unsigned v = 0;
        if (lane == 0 && *reinterpret_cast<volatile unsigned*>(G.inject)) v = atomicExch(G.inject, 0u);
        if (__shfl_sync(0xffffffffu, v, 0)) {
          ++it;
          continue;
        }
      }
      if (it >= NST) {
        const bool okw = lane == 0 ? mbar_wait(&empty[s], ph ^ 1u) : true;
        if (!__shfl_sync(0xffffffffu, okw, 0)) {
          if (lane == 0) atomicExch(kerr, 1u);
          break;
        }
      }
      unsigned char* st = smem + size_t(s) * G.stage_bytes;
      const uint32_t Z0 = 1 + stp.slab * Gp;
      // first lattice line / cell line and line counts of the ranges
      const uint32_t xl0 = stp.init ? stp.y - 1 : stp.y + 1, xnl = stp.init ? 2u : stp.nl;
      const uint32_t kl0 = stp.init ? stp.y - 1 : stp.y, knl = stp.init ? 1u : stp.nl;
      uint64_t lo = 0;
      uint32_t by = 0, dst = 0;
      const void* src = nullptr;
      const uint32_t q = uint32_t(lane);
      if (q < Gp + 2) {
        const uint32_t zp = Z0 - 1 + q;
        if (zp <= N) {
          widen<XT>((uint64_t(zp) * M1 + xl0) * M1, (uint64_t(zp) * M1 + xl0 + xnl - 1) * M1 + M1 - 1, lo, by);
          src = x + lo;
          dst = q * G.cap_x;
        }
      } else if (q < 2 * Gp + 3) {
        const uint32_t zc = Z0 - 1 + (q - (Gp + 2));
        if (zc < N && A.k) {
          widen<T>((uint64_t(zc) * N + kl0) * N, (uint64_t(zc) * N + kl0 + knl - 1) * N + N - 1, lo, by);
          src = A.k + lo;
          dst = off_k + (q - (Gp + 2)) * G.cap_k;
        }
      } else if (!stp.init && q < 2 * Gp + 3 + uint32_t(NS) * Gp) {
        const uint32_t i = (q - (2 * Gp + 3)) / Gp, g = (q - (2 * Gp + 3)) % Gp;
        const uint32_t z = Z0 + g;
        if (z <= W) {
          widen<T>((uint64_t(z) * M1 + stp.y) * M1, (uint64_t(z) * M1 + stp.y + stp.nl - 1) * M1 + M1 - 1, lo, by);
          src = (i == 0 ? st0 : st1) + lo;
          dst = off_s + (i * Gp + g) * G.cap_s;
        }
      }
      uint32_t total = by;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) total += __shfl_xor_sync(0xffffffffu, total, o);
      if (lane == 0) mbar_arrive_tx(&full[s], total);
      __syncwarp();
      if (by) bulk_g2s(st + dst, src, by, &full[s]);
      ++it;
    }
    // copies still in flight (none unless the consumers stopped early)
    if (lane == 0) {
      const uint32_t issued = it;
      for (uint32_t j = issued > NST ? issued - NST : 0; j < issued; ++j)
        if (!mbar_wait(&full[j % NST], (j / NST) & 1u)) atomicExch(kerr, 2u);
    }
    __syncwarp();
  } else {
    // ---------------- direct path first: the rows outside the slabs' interiors
    const bool skp = SE::skip(epi);
    acc += direct_rows<T, XT, Epi>(A, x, epi, st0, skp, M1, G.nbl_items, G.nbl_items + G.nedge_items,
                                   G.direct_masked != 0, blockIdx.x * NCW + warp, gridDim.x * NCW, lane);
    // ---------------- consumers
    const uint32_t tid = threadIdx.x;
    constexpr uint32_t PW = (W + CPT - 1) / CPT;  // threads per line
    const uint32_t grp = tid / PW, X = 1 + CPT * (tid - grp * PW);
    uint32_t it = 0;
    StreamIter<W, TY> sit(u0, u1);
    StreamStep stp;
    if constexpr (CPT == 2) {
      // window of 4 columns X-1..X+2 and 3 cells X-1, X, X+1: xp/xm [slot][column], kp [cell];
      // Kp / Km [slot][i]: i = 0, 2, 4 the cells, i = 1, 3 the sums of neighbouring cells, so row X
      // takes Kp[.][0..2] and columns 0..2, row X+1 takes Kp[.][2..4] and columns 1..3
      float2 xp2[3][4], Kp2[2][5];
      float xm2[3][4], Km2[2][5];
      const bool second = X + 1 <= W;  // the second row is an interior row
      while (sit.next(stp)) {
        const int s = int(it % NST);
        const uint32_t ph = (it / NST) & 1u;
        if (!mbar_wait(&full[s], ph)) {
          atomicExch(kerr, 3u);
          break;
        }
        const unsigned char* st = smem + size_t(s) * G.stage_bytes;
        const uint32_t Z0 = 1 + stp.slab * Gp, Z = Z0 + grp;
        if (grp < Gp && Z <= W) {
          const uint32_t xl0 = stp.init ? stp.y - 1 : stp.y + 1;
          const uint32_t kl0 = stp.init ? stp.y - 1 : stp.y;
          const float* xs[3];
#pragma unroll
          for (int q = 0; q < 3; ++q) {
            const uint64_t lo = (uint64_t(Z - 1 + q) * M1 + xl0) * M1;
            xs[q] = reinterpret_cast<const float*>(st + (grp + q) * G.cap_x) + (lo & (EX - 1)) + X;
          }
          const float* ks[2];
#pragma unroll
          for (int q = 0; q < 2; ++q) {
            const uint64_t lo = (uint64_t(Z - 1 + q) * N + kl0) * N;
            ks[q] = reinterpret_cast<const float*>(st + off_k + (grp + q) * G.cap_k) + (lo & (E - 1)) + (X - 1);
          }
          // cell sums of one cell line: cells X-1, X, X+1 paired over the cell planes Z-1 / Z
          auto cells = [&](int slot, int off) {
            float2 c[3];
#pragma unroll
            for (int e = 0; e < 3; ++e) c[e] = A.k ? make_float2(ks[0][off + e], ks[1][off + e]) : make_float2(1.f, 1.f);
            Kp2[slot][0] = c[0];
            Kp2[slot][2] = c[1];
            Kp2[slot][4] = c[2];
            Kp2[slot][1] = __fadd2_rn(c[0], c[1]);
            Kp2[slot][3] = __fadd2_rn(c[1], c[2]);
#pragma unroll
            for (int i = 0; i < 5; ++i) Km2[slot][i] = Kp2[slot][i].x + Kp2[slot][i].y;
          };
          if (stp.init) {
#pragma unroll
            for (int l = 0; l < 2; ++l)
#pragma unroll
              for (int d = 0; d < 4; ++d) {
                xp2[l][d] = make_float2(xs[0][l * int(M1) + d - 1], xs[2][l * int(M1) + d - 1]);
                xm2[l][d] = xs[1][l * int(M1) + d - 1];
              }
            cells(0, 0);
          } else {
            const uint64_t r0 = (uint64_t(Z) * M1 + stp.y) * M1;
            const float* ss = reinterpret_cast<const float*>(st + off_s + grp * G.cap_s) + (r0 & (E - 1)) + X;
            auto rows = [&](auto fast) {
              constexpr bool FAST = decltype(fast)::value;
#pragma unroll
              for (int j = 0; j < TY; ++j) {
                if (!FAST && uint32_t(j) >= stp.nl) break;
                const int a = j % 3, b = (j + 1) % 3, c = (j + 2) % 3, ka = j % 2, kb = (j + 1) % 2;
#pragma unroll
                for (int d = 0; d < 4; ++d) {
                  xp2[c][d] = make_float2(xs[0][j * int(M1) + d - 1], xs[2][j * int(M1) + d - 1]);
                  xm2[c][d] = xs[1][j * int(M1) + d - 1];
                }
                cells(kb, j * int(N));
                // (Kp[ka][2] + Kp[kb][2]) is S5's far-cell sum of row X and its near-cell sum of row X+1
                const float2 K2 = __fadd2_rn(Kp2[ka][2], Kp2[kb][2]);
#pragma unroll
                for (int o = 0; o < 2; ++o) {
                  // row X + o: columns o..o+2, cells Kp2[.][2o..2o+2]; the terms and order of the
                  // single-row packed form
                  const int i0 = 2 * o, i1 = 2 * o + 1, i2 = 2 * o + 2;
                  const float kc = Km2[ka][i1] + Km2[kb][i1];
                  const float2 K0 = o == 0 ? __fadd2_rn(Kp2[ka][i0], Kp2[kb][i0]) : K2;
                  const float2 Kf = o == 0 ? K2 : __fadd2_rn(Kp2[ka][i2], Kp2[kb][i2]);
                  float2 S5 = __fmul2_rn(K0, xp2[b][o]);
                  S5 = __ffma2_rn(Kf, xp2[b][o + 2], S5);
                  float2 S6 = __fmul2_rn(Kp2[ka][i1], xp2[a][o + 1]);
                  S6 = __ffma2_rn(Kp2[kb][i1], xp2[c][o + 1], S6);
                  float2 S7 = __fmul2_rn(Kp2[ka][i0], xp2[a][o]);
                  S7 = __ffma2_rn(Kp2[ka][i2], xp2[a][o + 2], S7);
                  S7 = __ffma2_rn(Kp2[kb][i0], xp2[c][o], S7);
                  S7 = __ffma2_rn(Kp2[kb][i2], xp2[c][o + 2], S7);
                  const float S0 = kc * xm2[b][o + 1];
                  float S3 = Km2[ka][i0] * xm2[a][o];
                  S3 += Km2[ka][i2] * xm2[a][o + 2];
                  S3 += Km2[kb][i0] * xm2[c][o];
                  S3 += Km2[kb][i2] * xm2[c][o + 2];
                  float sum = A.kr[0] * S0;
                  sum += A.kr[3] * S3;
                  sum += A.kr[5] * (S5.x + S5.y);
                  sum += A.kr[6] * (S6.x + S6.y);
                  sum += A.kr[7] * (S7.x + S7.y);
                  const float xc = xm2[b][o + 1];
                  const uint32_t row = uint32_t(r0) + uint32_t(j) * M1 + X + o;
                  T sv[1];
                  if (NS > 0) sv[0] = ss[j * int(M1) + o];
                  if (o == 0 || second) acc += SE::apply(epi, FAST ? false : skp, row, sum, xc, sv, false, kc);
                }
              }
            };
            if (!skp && A.k && stp.nl == uint32_t(TY)) rows(std::true_type{});
            else rows(std::false_type{});
          }
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[s]);
        ++it;
      }
    } else {
    // window: xp[slot][dx] pairs planes Z-1 / Z+1, xm[slot][dx] is plane Z, kp[slot][ex] pairs cell
    // planes Z-1 / Z (packed FP32 form); xw[plane][slot][dx], kw[cell plane][slot][ex] (scalar form)
    float2 xp[3][3], kp[2][2], Kp[2][3];
    T xm[3][3], Km[2][3];
    T xw[3][3][3], kw[2][2][2], K[2][3][3];
    while (sit.next(stp)) {
      const int s = int(it % NST);
      const uint32_t ph = (it / NST) & 1u;
      if (!mbar_wait(&full[s], ph)) {
        atomicExch(kerr, 3u);
        break;
      }
      const unsigned char* st = smem + size_t(s) * G.stage_bytes;
      const uint32_t Z0 = 1 + stp.slab * Gp, Z = Z0 + grp;
      const bool active = grp < Gp && Z <= W;
      if (active) {
        const uint32_t xl0 = stp.init ? stp.y - 1 : stp.y + 1;
        const uint32_t kl0 = stp.init ? stp.y - 1 : stp.y;
        // the thread's x planes Z-1, Z, Z+1 are ranges grp, grp+1, grp+2; line xl0 of each at xs[q]
        const XT* xs[3];
#pragma unroll
        for (int q = 0; q < 3; ++q) {
          const uint64_t lo = (uint64_t(Z - 1 + q) * M1 + xl0) * M1;
          xs[q] = reinterpret_cast<const XT*>(st + (grp + q) * G.cap_x) + (lo & (EX - 1)) + X;
        }
        const T* ks[2] = {nullptr, nullptr};
        if (A.k) {
#pragma unroll
          for (int q = 0; q < 2; ++q) {
            const uint64_t lo = (uint64_t(Z - 1 + q) * N + kl0) * N;
            ks[q] = reinterpret_cast<const T*>(st + off_k + (grp + q) * G.cap_k) + (lo & (E - 1)) + (X - 1);
          }
        }
        if (stp.init) {
          // x lines y-1 (slot 0) and y (slot 1), cell line y-1 (slot 0)
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
        } else {
          const uint64_t r0 = (uint64_t(Z) * M1 + stp.y) * M1;
          const T* ss = reinterpret_cast<const T*>(st + off_s + grp * G.cap_s) + (r0 & (E - 1)) + X;
          // FAST: a full stage with the coefficients given and the smoother running: rows
          // without a branch
          auto rows = [&](auto fast) {
            constexpr bool FAST = decltype(fast)::value;
#pragma unroll
            for (int j = 0; j < TY; ++j) {
              if (!FAST && uint32_t(j) >= stp.nl) break;
              // slots: x lines y+j-1, y+j, y+j+1 are a, b, c; cell lines y+j-1, y+j are ka, kb
              const int a = j % 3, b = (j + 1) % 3, c = (j + 2) % 3, ka = j % 2, kb = (j + 1) % 2;
              T sum, kc, xc;
              if constexpr (PK) {
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                  xp[c][d] = make_float2(xs[0][j * int(M1) + d - 1], xs[2][j * int(M1) + d - 1]);
                  xm[c][d] = xs[1][j * int(M1) + d - 1];
                }
#pragma unroll
                for (int cc = 0; cc < 2; ++cc)
                  kp[kb][cc] = (FAST || A.k) ? make_float2(ks[0][j * int(N) + cc], ks[1][j * int(N) + cc])
                                             : make_float2(1.f, 1.f);
                ksums2(kp[kb], Kp[kb], Km[kb]);
                kc = Km[ka][1] + Km[kb][1];  // the row's 8 cells
                // the terms of k_mf_q1_tiled's packed form, in its order
                float2 S5 = __fmul2_rn(__fadd2_rn(Kp[ka][0], Kp[kb][0]), xp[b][0]);
                S5 = __ffma2_rn(__fadd2_rn(Kp[ka][2], Kp[kb][2]), xp[b][2], S5);
                float2 S6 = __fmul2_rn(Kp[ka][1], xp[a][1]);
                S6 = __ffma2_rn(Kp[kb][1], xp[c][1], S6);
                float2 S7 = __fmul2_rn(Kp[ka][0], xp[a][0]);
                S7 = __ffma2_rn(Kp[ka][2], xp[a][2], S7);
                S7 = __ffma2_rn(Kp[kb][0], xp[c][0], S7);
                S7 = __ffma2_rn(Kp[kb][2], xp[c][2], S7);
                const T S0 = kc * xm[b][1];
                T S3 = Km[ka][0] * xm[a][0];
                S3 += Km[ka][2] * xm[a][2];
                S3 += Km[kb][0] * xm[c][0];
                S3 += Km[kb][2] * xm[c][2];
                sum = A.kr[0] * S0;
                sum += A.kr[3] * S3;
                sum += A.kr[5] * (S5.x + S5.y);
                sum += A.kr[6] * (S6.x + S6.y);
                sum += A.kr[7] * (S7.x + S7.y);
                xc = xm[b][1];
              } else {
#pragma unroll
                for (int q = 0; q < 3; ++q)
#pragma unroll
                  for (int d = 0; d < 3; ++d) xw[q][c][d] = T(xs[q][j * int(M1) + d - 1]);
                if (FAST || A.k) {
#pragma unroll
                  for (int q = 0; q < 2; ++q) {
                    kw[q][kb][0] = ks[q][j * int(N)];
                    kw[q][kb][1] = ks[q][j * int(N) + 1];
                  }
                } else {
#pragma unroll
                  for (int q = 0; q < 2; ++q) kw[q][kb][0] = kw[q][kb][1] = T(1);
                }
                ksums(kw, kb, K[kb]);
                kc = K[ka][1][1] + K[kb][1][1];
                // stencil form of the cell sum, the 6 face neighbours (coefficient 0) left out, as
                // in k_mf_q1_tiled: lines dy = 0, 1, 2 are slots a, b, c; cell lines ka (below), kb
                T S[8];
#pragma unroll
                for (int r = 0; r < 8; ++r) S[r] = T(0);
                const int sl[3] = {a, b, c};
#pragma unroll
                for (int dz = 0; dz < 3; ++dz)
#pragma unroll
                  for (int dy = 0; dy < 3; ++dy)
#pragma unroll
                    for (int dx = 0; dx < 3; ++dx) {
                      const int r = (dx != 1 ? 1 : 0) | (dy != 1 ? 2 : 0) | (dz != 1 ? 4 : 0);
                      if (r == 1 || r == 2 || r == 4) continue;
                      const T Kd = dy == 0 ? K[ka][dz][dx] : (dy == 2 ? K[kb][dz][dx] : K[ka][dz][dx] + K[kb][dz][dx]);
                      S[r] += Kd * xw[dz][sl[dy]][dx];
                    }
                sum = A.kr[0] * S[0];
#pragma unroll
                for (int r = 3; r < 8; ++r)
                  if (r != 4) sum += A.kr[r] * S[r];
                xc = xw[1][b][1];
              }
              const uint32_t row = uint32_t(r0) + uint32_t(j) * M1 + X;
              T sv[NS > 0 ? NS : 1];
              if (NS > 0) sv[0] = ss[j * int(M1)];
              if (NS > 1)
                sv[NS > 1 ? 1 : 0] =
                    reinterpret_cast<const T*>(reinterpret_cast<const unsigned char*>(ss) + Gp * G.cap_s)[j * int(M1)];
              acc += SE::apply(epi, FAST ? false : skp, row, sum, xc, sv, false, kc);
            }
          };
          if (!skp && A.k && stp.nl == uint32_t(TY)) rows(std::true_type{});
          else rows(std::false_type{});
        }
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(&empty[s]);
      ++it;
    }
    }
  }
  pdl_trigger();
  if (Epi::kReduce) {
    const double blk = block_sum<NT>(acc, sh);
    reduce_finish<NT>(blk, ws, counter, red_out, sh, false);
  }
}

// 8 consumer warps: two CTAs per SM at up to 96 registers
template<typename T, typename Epi, int NST, int MINB, int TY, int CM1, typename XT = T, int CPT = 1>
__global__ void __launch_bounds__(288, MINB)
    k_mf_q1_stream(MfView<T, 3> A, MfStream G, const XT* __restrict__ x, Epi epi, const T* st0, const T* st1,
                   double* ws, unsigned* counter, double* red_out, unsigned* kerr) {
  mf_stream_body<T, Epi, NST, TY, CM1, XT, 8, CPT>(A, G, x, epi, st0, st1, ws, counter, red_out, kerr);
}

// 16 consumer warps: one CTA per SM (544 threads; registers go to warps in groups of four, so the
// block is charged as 20 warps, 96 registers each)
template<typename T, typename Epi, int NST, int TY, int CM1, typename XT = T, int CPT = 1>
__global__ void __launch_bounds__(544, 1)
    k_mf_q1_stream16(MfView<T, 3> A, MfStream G, const XT* __restrict__ x, Epi epi, const T* st0, const T* st1,
                     double* ws, unsigned* counter, double* red_out, unsigned* kerr) {
  mf_stream_body<T, Epi, NST, TY, CM1, XT, 16, CPT>(A, G, x, epi, st0, st1, ws, counter, red_out, kerr);
}

// 12 consumer warps: one CTA per SM (416 threads, charged as 16 warps: 128 registers each), for the
// two-rows-per-thread form
template<typename T, typename Epi, int NST, int TY, int CM1, typename XT = T, int CPT = 1>
__global__ void __maxnreg__(128)
    k_mf_q1_stream12(MfView<T, 3> A, MfStream G, const XT* __restrict__ x, Epi epi, const T* st0, const T* st1,
                     double* ws, unsigned* counter, double* red_out, unsigned* kerr) {
  mf_stream_body<T, Epi, NST, TY, CM1, XT, 12, CPT>(A, G, x, epi, st0, st1, ws, counter, red_out, kerr);
}

}  // namespace fb
