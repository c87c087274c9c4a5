// Bulk-staged 3D Q1 restriction for structured levels whose filter is the lattice boundary.
//
// A tile is Lc consecutive interior coarse lines (Yc0..Yc0+Lc-1) of one interior coarse plane
// Zc, every interior point of each line. Its input is three contiguous fine ranges: the fine
// planes 2Zc-1, 2Zc, 2Zc+1, whole fine lines 2Yc0-1 .. 2(Yc0+Lc)-1 of each (a coarse point is
// the fine point with twice its coordinates, so no range needs clamping). One producer warp
// copies the three ranges of a tile with cp.async.bulk into an NST-deep ring of stages
// (ranges widened to 16-byte boundaries, which the 64 bytes of slack of every device
// allocation allow); eight consumer warps form the coarse rows: G groups of Wc threads (one
// per interior coarse point of a line) walk TYC coarse lines each and keep the fine line two
// coarse lines share in registers (18 new fine values per coarse row).
//
// Interior coarse points meet all 27 fine neighbours with weights 1/2, 1, 1/2 per axis; the
// terms and their order are those of k_rest_q1 (the products of powers of two are exact), so
// the result equals that kernel's bit for bit. The coarse boundary rows are filtered, hence
// zero: the consumers write them through the epilogue before their first tile.
//
// Every mbarrier wait is bounded as in k_mf_q1_tiled; on expiry the kernel records it in
// `kerr`, stops taking tiles, waits (bounded) for its copies in flight and returns.
#pragma once
#include "fb_mf.cuh"

namespace fb {

// G describes the coarse lattice: M1 = Mc1, Lt = Lc, G = groups, tpp / ntiles / dz / dyt as
// for the operator tiles, cap_x = bytes reserved per fine range, nbl_items / nedge_items the
// direct items of the coarse boundary.
template<typename T, int NST, int TYC>
__global__ void __launch_bounds__(288, 1) k_rest_q1_staged(MfTile G, uint32_t Mf1, const T* __restrict__ xf,
                                                           EpiRestrict<T> epi, double* ws, unsigned* counter,
                                                           double* red_out, unsigned* kerr) {
  constexpr uint64_t E = 16 / sizeof(T);
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
  const uint32_t Mc1 = G.M1, Wc = Mc1 - 2;
  double acc = 0.0;
  if (warp == 8) {
    // ---------------- producer: lane q < 3 copies fine plane 2 Zc - 1 + q of the tile
    uint32_t it = 0;
    TileIter ti(G, blockIdx.x);
    for (uint32_t t = blockIdx.x; t < G.ntiles; t += gridDim.x, ++it, ti.next(G)) {
      const int s = int(it % NST);
      const uint32_t ph = (it / NST) & 1u;
      if (it >= NST) {
        const bool okw = lane == 0 ? mbar_wait(&empty[s], ph ^ 1u) : true;
        if (!__shfl_sync(0xffffffffu, okw, 0)) {
          if (lane == 0) atomicExch(kerr, 1u);
          break;
        }
      }
      const TileGeo g = tile_geo(G, ti);
      uint64_t lo = 0;
      uint32_t by = 0;
      if (lane < 3) {
        const uint64_t fz = 2 * uint64_t(g.Z) - 1 + lane;
        widen<T>((fz * Mf1 + 2 * g.Y0 - 1) * Mf1, (fz * Mf1 + 2 * (g.Y0 + g.lt) - 1) * Mf1 + Mf1 - 1, lo, by);
      }
      uint32_t total = by;
#pragma unroll
      for (int o = 2; o > 0; o >>= 1) total += __shfl_xor_sync(0xffffffffu, total, o);
      if (lane == 0) mbar_arrive_tx(&full[s], total);
      __syncwarp();
      if (by) bulk_g2s(smem + size_t(s) * G.stage_bytes + lane * G.cap_x, xf + lo, by, &full[s]);
    }
    // copies still in flight (none unless the consumers stopped early)
    if (lane == 0) {
      const uint32_t issued = it;
      for (uint32_t j = issued > NST ? issued - NST : 0; j < issued; ++j)
        if (!mbar_wait(&full[j % NST], (j / NST) & 1u)) atomicExch(kerr, 2u);
    }
    __syncwarp();
  } else {
    // ---------------- coarse boundary rows (filtered: zero), while the first copies fly
    for (uint32_t item = blockIdx.x * 8 + warp; item < G.nbl_items + G.nedge_items; item += gridDim.x * 8) {
      uint32_t X, Y, Z;
      const int32_t row = direct_row(item, lane, Mc1, G.nbl_items, X, Y, Z);
      if (row >= 0) {
        epi.rhs[row] = T(0);
        if (epi.sol1) epi.sol1[row] = T(0);
      }
    }
    // ---------------- consumers: TYC coarse rows per thread and tile
    EpiRestrict<T> ei = epi;
    ei.mask = nullptr;  // tile rows are interior: never filtered
    const uint32_t tid = threadIdx.x;
    const uint32_t grp = tid / Wc, Xc = 1 + (tid - grp * Wc);
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
      const uint32_t l0 = grp * TYC;  // first coarse line of this group, relative to Yc0
      if (active && l0 < g.lt) {
        // fine column 2 Xc of fine line 2 (Yc0 + l0) - 1 in each staged plane
        const T* fp[3];
#pragma unroll
        for (int q = 0; q < 3; ++q) {
          const uint64_t fz = 2 * uint64_t(g.Z) - 1 + q;
          const uint64_t flo = (fz * Mf1 + 2 * g.Y0 - 1) * Mf1;
          fp[q] = reinterpret_cast<const T*>(st + q * G.cap_x) + (flo & (E - 1)) + 2 * l0 * Mf1 + 2 * Xc;
        }
        // window v[fine plane][fine line][fine column], offsets -1, 0, +1 from the coarse point
        T v[3][3][3];
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
          for (int c = 0; c < 3; ++c) v[a][0][c] = fp[a][c - 1];
        const uint32_t row0 = (g.Z * Mc1 + g.Y0 + l0) * Mc1 + Xc;
        // the epilogue's inverse diagonal of the thread's rows, loaded together before the window
        // (one at a time, each row's epilogue waited for its load)
        T idv[TYC];
#pragma unroll
        for (int j = 0; j < TYC; ++j) idv[j] = (ei.sol1 && l0 + j < g.lt) ? __ldg(ei.invd + row0 + j * Mc1) : T(0);
#pragma unroll
        for (int j = 0; j < TYC; ++j) {
          if (l0 + j >= g.lt) break;
#pragma unroll
          for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int b = 1; b < 3; ++b)
#pragma unroll
              for (int c = 0; c < 3; ++c) v[a][b][c] = fp[a][(2 * j + b) * int(Mf1) + c - 1];
          T s = T(0);
#pragma unroll
          for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int b = 0; b < 3; ++b)
#pragma unroll
              for (int c = 0; c < 3; ++c) {
                const T w = (b == 1 ? T(1) : T(0.5)) * (c == 1 ? T(1) : T(0.5)) * (a == 1 ? T(1) : T(0.5));
                s += w * v[a][b][c];
              }
          acc += ei.with_invd(row0 + j * Mc1, s, idv[j]);
#pragma unroll
          for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int c = 0; c < 3; ++c) v[a][0][c] = v[a][2][c];
        }
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(&empty[s]);
    }
  }
  pdl_trigger();
  const double blk = block_sum<288>(acc, sh);
  reduce_finish<288>(blk, ws, counter, red_out, sh, false);
}

}  // namespace fb
