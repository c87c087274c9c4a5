// Streaming form of the packed stencil SpMV (FP16 or FP32 stencil values, k_stencil_packed's
// storage) on the 257^3 level of a structured 3D Q1 hierarchy whose filter is the lattice
// boundary, with the epilogues of the staged kernels.
//
// k_stencil_packed gathers the 27 neighbours of every row from x through L1/L2, one load per
// neighbour; here x is staged in shared memory as in k_mf_q1_stream (slabs of G interior planes,
// one contiguous range of slab-lines per CTA, each line of x and of the streamed epilogue inputs
// copied once per run with cp.async.bulk into an NST-deep mbarrier ring) and every consumer
// thread walks up its column with a sliding 3x3x3 register window of x, so a row costs 9 shared
// loads of the new line plus its own 8-byte stencil-value loads from global memory (coalesced
// across the warp's consecutive rows, issued one row ahead). The 27 products are summed in slot
// order, as in k_stencil_packed, so the rows' products and epilogues are bit-identical with it
// (the reductions group their partial sums differently). The rows outside the slabs' interiors all
// lie on the lattice boundary and are filtered: their epilogues run without the product.
#pragma once
#include "fb_mf_stream.cuh"

namespace fb {

struct StStream {
  uint32_t G;                      // planes per slab
  uint32_t nslab;                  // ceil(W / G)
  uint64_t units;                  // nslab * W slab-lines
  uint32_t cap_x, cap_s;           // bytes reserved per x / stream range in a stage
  uint32_t stage_bytes;
  uint32_t nbl_items, nedge_items; // rows outside the slab interiors, as MfTile
  float scale;                     // FP16 values: the level's scale
  unsigned* inject;                // test hook, as MfTile
};

template<typename VT, typename Epi, int NST, int TY, int CM1, int NCW>
__global__ void __launch_bounds__(32 * (NCW + 1), 1)
    k_stencil_stream(StStream G, const VT* __restrict__ val, const float* __restrict__ x, Epi epi, const float* st0,
                     const float* st1, double* ws, unsigned* counter, double* red_out, unsigned* kerr) {
  static_assert(TY % 3 == 0, "x line slots repeat every 3 rows");
  constexpr int NT = 32 * (NCW + 1);
  using SE = Staged<Epi>;
  constexpr int NS = SE::kStreams;
  constexpr uint32_t M1 = CM1, N = M1 - 1, W = M1 - 2;
  constexpr int PW = Pack8<VT>::W;        // stencil values per 8-byte load
  constexpr int NG = (27 + PW - 1) / PW;  // 8-byte loads per row
  constexpr uint64_t E = 4;               // floats per 16 bytes
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
  // stage layout: (G+2) x planes | NS * G stream planes
  const uint32_t off_s = (Gp + 2) * G.cap_x;
  const uint64_t u0 = G.units * blockIdx.x / gridDim.x, u1 = G.units * (blockIdx.x + 1) / gridDim.x;
  double acc = 0.0;
  if (warp == NCW) {
    // ---------------- producer: lane q issues range q (0..G+1: x planes Z0-1..Z0+G; then the streams)
    uint32_t it = 0;
    StreamIter<W, TY> sit(u0, u1);
    StreamStep stp;
    while (sit.next(stp)) {
      const int s = int(it % NST);
      const uint32_t ph = (it / NST) & 1u;
      if (G.inject && it == 0 && blockIdx.x == 0) {
        // test hook: nothing arrives on this stage, so the consumers' bounded wait on it expires
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
      const uint32_t xl0 = stp.init ? stp.y - 1 : stp.y + 1, xnl = stp.init ? 2u : stp.nl;
      uint64_t lo = 0;
      uint32_t by = 0, dst = 0;
      const void* src = nullptr;
      const uint32_t q = uint32_t(lane);
      if (q < Gp + 2) {
        const uint32_t zp = Z0 - 1 + q;
        if (zp <= N) {
          widen<float>((uint64_t(zp) * M1 + xl0) * M1, (uint64_t(zp) * M1 + xl0 + xnl - 1) * M1 + M1 - 1, lo, by);
          src = x + lo;
          dst = q * G.cap_x;
        }
      } else if (!stp.init && q < Gp + 2 + uint32_t(NS) * Gp) {
        const uint32_t i = (q - (Gp + 2)) / Gp, g = (q - (Gp + 2)) % Gp;
        const uint32_t z = Z0 + g;
        if (z <= W) {
          widen<float>((uint64_t(z) * M1 + stp.y) * M1, (uint64_t(z) * M1 + stp.y + stp.nl - 1) * M1 + M1 - 1, lo, by);
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
    // ---------------- the rows outside the slabs' interiors (all filtered)
    const bool skp = SE::skip(epi);
    const MfView<float, 3> none{};
    acc += direct_rows<float, float, Epi>(none, x, epi, st0, skp, M1, G.nbl_items, G.nbl_items + G.nedge_items, true,
                                          blockIdx.x * NCW + warp, gridDim.x * NCW, lane);
    // ---------------- consumers: window xw[plane Z-1..Z+1][line slot][column X-1..X+1]
    const uint32_t tid = threadIdx.x;
    const uint32_t grp = tid / W, X = 1 + (tid - grp * W);
    float xw[3][3][3];
    uint32_t it = 0;
    StreamIter<W, TY> sit(u0, u1);
    StreamStep stp;
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
        const float* xs[3];
#pragma unroll
        for (int q = 0; q < 3; ++q) {
          const uint64_t lo = (uint64_t(Z - 1 + q) * M1 + xl0) * M1;
          xs[q] = reinterpret_cast<const float*>(st + (grp + q) * G.cap_x) + (lo & (E - 1)) + X;
        }
        if (stp.init) {
#pragma unroll
          for (int q = 0; q < 3; ++q)
#pragma unroll
            for (int l = 0; l < 2; ++l)
#pragma unroll
              for (int d = 0; d < 3; ++d) xw[q][l][d] = xs[q][l * int(M1) + d - 1];
        } else {
          const uint64_t r0 = (uint64_t(Z) * M1 + stp.y) * M1;
          const float* ss = reinterpret_cast<const float*>(st + off_s + grp * G.cap_s) + (r0 & (E - 1)) + X;
          // the packed values of row r: 8-byte loads g = 0..NG-1 at vrow(r) + g * 32 * PW; each row's
          // loads are issued one row ahead, so two rows' loads are in flight per thread
          auto vrow = [&](uint32_t r) { return val + (size_t(r >> 5) * NG * 32 + (r & 31)) * PW; };
          uint2 nraw[NG];
          {
            const VT* vp = vrow(uint32_t(r0) + X);
#pragma unroll
            for (int g = 0; g < NG; ++g) nraw[g] = Pack8<VT>::raw(vp + g * 32 * PW);
          }
#pragma unroll
          for (int j = 0; j < TY; ++j) {
            if (uint32_t(j) >= stp.nl) break;
            uint2 craw[NG];
#pragma unroll
            for (int g = 0; g < NG; ++g) craw[g] = nraw[g];
            if (j + 1 < TY && uint32_t(j + 1) < stp.nl) {
              const VT* vq = vrow(uint32_t(r0) + uint32_t(j + 1) * M1 + X);
#pragma unroll
              for (int g = 0; g < NG; ++g) nraw[g] = Pack8<VT>::raw(vq + g * 32 * PW);
            }
            // x lines y+j-1, y+j, y+j+1 are slots a, b, c
            const int a = j % 3, b = (j + 1) % 3, c = (j + 2) % 3;
#pragma unroll
            for (int q = 0; q < 3; ++q)
#pragma unroll
              for (int d = 0; d < 3; ++d) xw[q][c][d] = xs[q][j * int(M1) + d - 1];
            const uint32_t row = uint32_t(r0) + uint32_t(j) * M1 + X;
            float sum = 0.0f;
#pragma unroll
            for (int g = 0; g < NG; ++g) {
              float v[PW];
              Pack8<VT>::cvt(craw[g], v);
#pragma unroll
              for (int e = 0; e < PW; ++e) {
                const int k = g * PW + e;  // slot k = (dz+1)*9 + (dy+1)*3 + (dx+1)
                if (k < 27) {
                  const int dz = k / 9, dy = (k / 3) % 3, dx = k % 3;
                  const int sl = dy == 0 ? a : (dy == 1 ? b : c);
                  sum += v[e] * xw[dz][sl][dx];
                }
              }
            }
            if (sizeof(VT) == 2) sum *= G.scale;
            float sv[NS > 0 ? NS : 1];
            if (NS > 0) sv[0] = ss[j * int(M1)];
            if (NS > 1)
              sv[NS > 1 ? 1 : 0] =
                  reinterpret_cast<const float*>(reinterpret_cast<const unsigned char*>(ss) + Gp * G.cap_s)[j * int(M1)];
            acc += SE::apply(epi, skp, row, sum, xw[1][b][1], sv, false, 0.0f);
          }
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
