// Streaming form of the matrix-free Q1 operator on the two finest structured 3D levels
// (lattice size a compile-time constant), with the epilogues of k_mf_q1_tiled.
//
// The interior planes form slabs of G consecutive planes, one thread group of W = M1 - 2 threads
// per plane and one thread per interior point X of a line. The slab-lines (slab, interior line Y)
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
// to 16-byte boundaries, which the padded allocations allow); NCW (8 or 16) consumer warps compute. Rows
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

// NCW consumer warps (8 or 16) and one producer warp per CTA
template<typename T, typename Epi, int NST, int MINB, int TY, int CM1, typename XT = T, int NCW = 8>
__global__ void __launch_bounds__(32 * (NCW + 1), MINB)
    k_mf_q1_stream(MfView<T, 3> A, MfStream G, const XT* __restrict__ x, Epi epi, const T* st0, const T* st1,
                   double* ws, unsigned* counter, double* red_out, unsigned* kerr) {
  static_assert(TY % 6 == 0, "window slots repeat every 6 rows");
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
    // ---------------- direct path first: boundary lines and the end points of interior lines
    {
      const uint32_t cpl = (M1 + 31) / 32;
      const uint32_t nitems = G.nbl_items + G.nedge_items;
      for (uint32_t item = blockIdx.x * NCW + warp; item < nitems; item += gridDim.x * NCW) {
        int32_t row = -1;
        uint32_t X = 0, Y = 0, Z = 0;
        if (item < G.nbl_items) {
          const uint32_t bl = item / cpl;
          X = (item - bl * cpl) * 32 + lane;
          if (bl < 2 * M1) { Z = bl < M1 ? 0 : M1 - 1; Y = bl < M1 ? bl : bl - M1; }
          else { const uint32_t r = bl - 2 * M1; Z = 1 + (r >> 1); Y = (r & 1) ? M1 - 1 : 0; }
          if (X < M1) row = int32_t((Z * M1 + Y) * M1 + X);
        } else {
          const uint32_t li = (item - G.nbl_items) * 16 + (lane >> 1);
          if (li < W * W) {
            const uint32_t zq = li / W;
            Y = 1 + (li - zq * W); Z = 1 + zq;
            X = (lane & 1) ? M1 - 1 : 0;
            row = int32_t((Z * M1 + Y) * M1 + X);
          }
        }
        if (row >= 0) {
          const T s = G.direct_masked ? T(0) : mf_row_direct<T, XT>(A, x, row, int32_t(X), int32_t(Y), int32_t(Z));
          acc += epi(uint32_t(row), s);
        }
      }
    }
    // ---------------- consumers
    const bool skp = SE::skip(epi);
    const uint32_t tid = threadIdx.x;
    const uint32_t grp = tid / W, X = 1 + (tid - grp * W);
    uint32_t it = 0;
    StreamIter<W, TY> sit(u0, u1);
    StreamStep stp;
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
  pdl_trigger();
  if (Epi::kReduce) {
    const double blk = block_sum<NT>(acc, sh);
    reduce_finish<NT>(blk, ws, counter, red_out, sh, false);
  }
}

}  // namespace fb
