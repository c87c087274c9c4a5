// The coarse end of the V-cycle in one launch: all levels from the first one with at most a
// few ten thousand rows down to the coarsest, on one thread-block cluster.
//
// On those levels every operation of the V-cycle is a few microseconds of launch latency
// and tail for a few microseconds of work. Here one cluster of CS CTAs runs the same
// operation sequence as the per-operation kernels (smoothing steps, defect, restriction,
// coarse solve, prolongation, post-smoothing, with the same skip tests and reductions) and
// separates dependent steps with cluster barriers (barrier.cluster, release/acquire).
// Values written inside the kernel are read with ld.global.cg (L2), so no SM reads a stale
// L1 line of another SM's result. Reductions are deterministic: one partial per CTA, summed
// in rank order by every thread after the barrier. The operator is the matrix-free Q1 one
// (structured hierarchies, FB_FORMAT_MATFREE); the per-row arithmetic is that of k_mf_q1,
// k_rest_q1(_3d), k_prol_q1(_3d), k_dense_solve and the Jacobi/defect/restriction epilogues.
#pragma once
#include <cooperative_groups.h>

#include "fb_mf.cuh"

namespace fb {

template<typename T>
struct CLevel {
  uint32_t n, M1;        // rows, lattice points per side
  const T* k;            // per-cell coefficient (nullptr = 1)
  T kr[8];               // (h/2)^(dim-2) K_ref[0][r]
  const uint32_t* mask;  // Dirichlet bit mask
  const T* invd;         // omega_J / diag
  T *rhs, *x, *y, *def;
  double *bn, *dn;       // ||rhs||^2 and ||first post-smoothing defect||^2 of this level
};

constexpr int kCoarseMax = 8;

template<typename T>
struct CoarseArgs {
  CLevel<T> L[kCoarseMax];  // L[0] = first fused level, L[nlv-1] = coarsest
  int nlv, nu, coarse;
  T omega;
  const T* cinv;            // dense inverse of the coarsest filtered system (FB_COARSE_DIRECT)
  int s1_coarsest;          // the restriction onto the coarsest level forms its first smoothing step
};

template<typename T> __device__ __forceinline__ T ldc(const T* p) { return __ldcg(p); }

// A(k) x for one row (clamped gathers, cells outside the domain skipped), x read through L2
template<typename T, int DIM>
__device__ __forceinline__ T coarse_row(const CLevel<T>& L, const T* x, int32_t row) {
  constexpr int S = DIM == 3 ? 27 : 9;
  const int32_t last = int32_t(L.n) - 1;
  const int32_t M1 = int32_t(L.M1), N = M1 - 1;
  T xv[S];
#pragma unroll
  for (int j = 0; j < S; ++j) {
    const int dx = j % 3 - 1, dy = (j / 3) % 3 - 1, dz = DIM == 3 ? j / 9 - 1 : 0;
    int32_t col = row + (dz * M1 + dy) * M1 + dx;
    col = col < 0 ? 0 : (col > last ? last : col);
    xv[j] = ldc(x + col);
  }
  const int32_t X = row % M1, t = row / M1;
  const int32_t Y = DIM == 3 ? t % M1 : t, Z = DIM == 3 ? t / M1 : 0;
  T s = T(0);
#pragma unroll
  for (int e = 0; e < (1 << DIM); ++e) {
    const int ox = e & 1, oy = (e >> 1) & 1, oz = (e >> 2) & 1;
    const int a = (1 - ox) | ((1 - oy) << 1) | (DIM == 3 ? (1 - oz) << 2 : 0);
    const int32_t ex = X - 1 + ox, ey = Y - 1 + oy, ez = DIM == 3 ? Z - 1 + oz : 0;
    const bool valid = uint32_t(ex) < uint32_t(N) && uint32_t(ey) < uint32_t(N) &&
                       (DIM == 2 || uint32_t(ez) < uint32_t(N));
    const int64_t eidx = valid ? int64_t(ex) + int64_t(N) * (ey + int64_t(N) * ez) : 0;
    T ke = L.k ? __ldg(L.k + eidx) : T(1);
    ke = valid ? ke : T(0);
    T in = T(0);
#pragma unroll
    for (int b = 0; b < (1 << DIM); ++b) {
      const int dx = ox - 1 + (b & 1), dy = oy - 1 + ((b >> 1) & 1);
      const int dz = DIM == 3 ? oz - 1 + ((b >> 2) & 1) : 0;
      const int j = DIM == 3 ? (dz + 1) * 9 + (dy + 1) * 3 + (dx + 1) : (dy + 1) * 3 + (dx + 1);
      in += L.kr[a ^ b] * xv[j];
    }
    s += ke * in;
  }
  return s;
}

// restriction R d at coarse row i of level C from fine level F (k_rest_q1 arithmetic)
template<typename T, int DIM>
__device__ __forceinline__ T coarse_rest(const CLevel<T>& F, const CLevel<T>& C, const T* xf, uint32_t i) {
  const int Mc1 = int(C.M1), Mf1 = int(F.M1);
  const int X = int(i) % Mc1, t = int(i) / Mc1;
  const int Y = DIM == 3 ? t % Mc1 : t, Z = DIM == 3 ? t / Mc1 : 0;
  const int Fm = Mf1 - 1, Fz = DIM == 3 ? Fm : 0;
  int fx[3], fy[3], fz[3];
  T wx[3], wy[3], wz[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const int ox = 2 * X + d - 1, oy = 2 * Y + d - 1, oz = 2 * Z + d - 1;
    const T wd = d == 1 ? T(1) : T(0.5);
    wx[d] = (ox < 0 || ox > Fm) ? T(0) : wd;
    wy[d] = (oy < 0 || oy > Fm) ? T(0) : wd;
    wz[d] = DIM == 3 ? ((oz < 0 || oz > Fz) ? T(0) : wd) : (d == 1 ? T(1) : T(0));
    fx[d] = ox < 0 ? 0 : (ox > Fm ? Fm : ox);
    fy[d] = oy < 0 ? 0 : (oy > Fm ? Fm : oy);
    fz[d] = oz < 0 ? 0 : (oz > Fz ? Fz : oz);
  }
  T s = T(0);
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      const T* row = xf + (size_t(fz[a]) * Mf1 + fy[b]) * Mf1;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const T v = (DIM == 3 || a == 1) ? ldc(row + fx[c]) : T(0);
        s += (wx[c] * wy[b] * wz[a]) * v;
      }
    }
  return s;
}

// prolongation P x_c at fine row i of level F from coarse level C (k_prol_q1 arithmetic)
template<typename T, int DIM>
__device__ __forceinline__ T coarse_prol(const CLevel<T>& F, const CLevel<T>& C, const T* xc, uint32_t i) {
  const uint32_t Mf1 = F.M1, Mc1 = C.M1;
  const uint32_t X = i % Mf1, t = i / Mf1;
  const uint32_t Y = DIM == 3 ? t % Mf1 : t, Z = DIM == 3 ? t / Mf1 : 0;
  const uint32_t cx0 = X >> 1, cx1 = (X + 1) >> 1, cy0 = Y >> 1, cy1 = (Y + 1) >> 1;
  const uint32_t cz0 = Z >> 1, cz1 = (Z + 1) >> 1;
  const T w = ((X & 1) ? T(0.5) : T(1)) * ((Y & 1) ? T(0.5) : T(1)) * ((Z & 1) ? T(0.5) : T(1));
  const T wx1 = (X & 1) ? w : T(0), wy1 = (Y & 1) ? T(1) : T(0), wz1 = (Z & 1) ? T(1) : T(0);
  const size_t r00 = (size_t(cz0) * Mc1 + cy0) * Mc1, r01 = (size_t(cz0) * Mc1 + cy1) * Mc1;
  T s = T(0);
  s += w * ldc(xc + r00 + cx0);
  s += wx1 * ldc(xc + r00 + cx1);
  s += (wy1 * w) * ldc(xc + r01 + cx0);
  s += (wy1 * wx1) * ldc(xc + r01 + cx1);
  if (DIM == 3) {
    const size_t r10 = (size_t(cz1) * Mc1 + cy0) * Mc1, r11 = (size_t(cz1) * Mc1 + cy1) * Mc1;
    s += (wz1 * w) * ldc(xc + r10 + cx0);
    s += (wz1 * wx1) * ldc(xc + r10 + cx1);
    s += (wz1 * wy1 * w) * ldc(xc + r11 + cx0);
    s += (wz1 * wy1 * wx1) * ldc(xc + r11 + cx1);
  }
  return s;
}

// a row's smoothing inputs (its x, rhs and inverse diagonal values and its filter bit), loaded
// before the row's product so that they do not wait behind its gathers
template<typename T>
struct RowIn {
  T xc, b, id;
  bool m;
};
template<typename T>
__device__ __forceinline__ RowIn<T> row_in(const CLevel<T>& L, const T* cur, const T* b, uint32_t i) {
  return {ldc(cur + i), ldc(b + i), __ldg(L.invd + i), masked(L.mask, i)};
}

// one Jacobi step at a row from the product s (EpiJacobi without skip)
template<typename T>
__device__ __forceinline__ T jacobi_row(T om, const RowIn<T>& in, T s) {
  const T d = in.b - s;
  return in.m ? in.xc : om * (in.id * d) + in.xc;
}

// post-smoothing step at a row (EpiJacobi with s0 = o0 and skip test; the first step reduces
// ||d||^2)
template<typename T>
__device__ __forceinline__ T post_row(T om, const RowIn<T>& in, T o0, T s, bool skip, bool first, double& acc) {
  if (skip) return o0;
  const T d = in.b - s;
  if (in.m) return in.xc;
  if (first) acc += double(d) * double(d);
  return om * (in.id * d) + in.xc;
}

// deterministic cluster-wide sum; ends with a cluster barrier, result in every thread. Each CTA
// stores its partial into slot [its rank] of every CTA's shared array part (distributed shared
// memory), so after the barrier the partials are summed in rank order from local shared memory.
// part is double-buffered by the caller (consecutive sums use alternate halves), so a CTA that
// runs ahead into the next sum never overwrites a partial that a slower CTA has still to read.
template<int THREADS>
__device__ __forceinline__ double cluster_sum(double v, double* part, double* sh,
                                              cooperative_groups::cluster_group& cl) {
  const double blk = block_sum<THREADS>(v, sh);
  const uint32_t nb = cl.num_blocks(), me = cl.block_rank();
  if (threadIdx.x == 0)
    for (uint32_t r = 0; r < nb; ++r) *cl.map_shared_rank(part + me, r) = blk;
  cl.sync();
  double t = 0.0;
  for (uint32_t r = 0; r < nb; ++r) t += part[r];
  return t;
}

template<typename T, int DIM, int THREADS>
__global__ void __launch_bounds__(THREADS, 1) k_coarse_cycle(CoarseArgs<T> A) {
  namespace cgr = cooperative_groups;
  pdl_wait();
  // the cluster uses 16 SMs: let the next kernel's CTAs take the others (they wait for us)
  pdl_trigger();
  cgr::cluster_group cl = cgr::this_cluster();
  __shared__ double sh[THREADS / 32];
  __shared__ double part[2][16];  // cluster partials, double-buffered
  const uint32_t gt = cl.block_rank() * THREADS + threadIdx.x;
  const uint32_t gs = cl.num_blocks() * THREADS;
  const int nu = A.nu;
  const T om = A.omega;
  int rk = 0;  // reductions so far (double-buffered scratch)
  T* sol[kCoarseMax];
  double bnorm = *((volatile const double*)A.L[0].bn);  // formed by the launch before this one
  // ---------------- descent (multigrid.hpp:1711-1832)
  for (int l = 0; l + 1 < A.nlv; ++l) {
    const CLevel<T>& L = A.L[l];
    const T* b = L.rhs;
    const double bv = sqrt(bnorm);
    const bool skip = !isfinite(bv) || bv <= double(eps_of<T>()) * double(eps_of<T>());
    T* cur = L.x;
    T* oth = L.y;
    if (nu < 2) {
      for (uint32_t i = gt; i < L.n; i += gs)
        cur[i] = (skip || masked(L.mask, i)) ? T(0) : om * (__ldg(L.invd + i) * ldc(b + i));
      cl.sync();
    }
    for (int it = 1; it < nu; ++it) {
      for (uint32_t i = gt; i < L.n; i += gs) {
        const RowIn<T> in = row_in(L, cur, b, i);  // ahead of the row's gathers
        const T s = coarse_row<T, DIM>(L, cur, int32_t(i));
        oth[i] = skip ? T(0) : jacobi_row(om, in, s);
      }
      cl.sync();
      T* tmp = cur; cur = oth; oth = tmp;
    }
    sol[l] = cur;
    for (uint32_t i = gt; i < L.n; i += gs) {
      const T bi = ldc(b + i);
      const bool mk = masked(L.mask, i);
      const T s = coarse_row<T, DIM>(L, cur, int32_t(i));
      L.def[i] = mk ? T(0) : bi - s;
    }
    cl.sync();
    const CLevel<T>& C = A.L[l + 1];
    const bool s1 = nu >= 2 && (l + 2 < A.nlv || A.s1_coarsest);
    double acc = 0.0;
    for (uint32_t i = gt; i < C.n; i += gs) {
      const bool mk = masked(C.mask, i);
      const T id = s1 ? __ldg(C.invd + i) : T(0);  // ahead of the restriction's loads
      const T v = mk ? T(0) : coarse_rest<T, DIM>(L, C, L.def, i);
      C.rhs[i] = v;
      if (s1) C.x[i] = mk ? T(0) : om * (id * v);
      acc += double(v) * double(v);
    }
    bnorm = cluster_sum<THREADS>(acc, part[rk++ & 1], sh, cl);
    if (gt == 0) *C.bn = bnorm;
  }
  // ---------------- coarsest level (multigrid.hpp:1524-1587)
  {
    const int l = A.nlv - 1;
    const CLevel<T>& L = A.L[l];
    const T* b = L.rhs;
    if (A.coarse == FB_COARSE_DIRECT) {
      const uint32_t lane = gt & 31;
      for (uint32_t row = gt >> 5; row < L.n; row += gs >> 5) {
        double s = 0.0;
        for (uint32_t j = lane; j < L.n; j += 32) s += double(__ldg(A.cinv + uint64_t(row) * L.n + j)) * double(ldc(b + j));
        s = warp_sum(s);
        if (lane == 0) L.x[row] = T(s);
      }
      cl.sync();
      sol[l] = L.x;
    } else if (A.coarse == FB_COARSE_SMOOTHER) {
      const double bv = sqrt(bnorm);
      const bool skip = !isfinite(bv) || bv <= double(eps_of<T>()) * double(eps_of<T>());
      T* cur = L.x;
      T* oth = L.y;
      if (nu < 2) {
        for (uint32_t i = gt; i < L.n; i += gs)
          cur[i] = (skip || masked(L.mask, i)) ? T(0) : om * (__ldg(L.invd + i) * ldc(b + i));
        cl.sync();
      }
      for (int it = 1; it < nu; ++it) {
        for (uint32_t i = gt; i < L.n; i += gs) {
          const T s = coarse_row<T, DIM>(L, cur, int32_t(i));
          T o;
          if (skip) o = T(0);
          else {
            const T xc = ldc(cur + i);
            const T d = ldc(b + i) - s;
            o = masked(L.mask, i) ? xc : om * (__ldg(L.invd + i) * d) + xc;
          }
          oth[i] = o;
        }
        cl.sync();
        T* tmp = cur; cur = oth; oth = tmp;
      }
      sol[l] = cur;
    } else {  // FB_COARSE_NONE: x = filter_cor(b)
      for (uint32_t i = gt; i < L.n; i += gs) L.x[i] = masked(L.mask, i) ? T(0) : ldc(b + i);
      cl.sync();
      sol[l] = L.x;
    }
  }
  // ---------------- ascent (multigrid.hpp:1843-2000)
  for (int l = A.nlv - 2; l >= 0; --l) {
    const CLevel<T>& L = A.L[l];
    const CLevel<T>& C = A.L[l + 1];
    const T* b = L.rhs;
    T* cur = sol[l];
    T* oth = (cur == L.x) ? L.y : L.x;
    for (uint32_t i = gt; i < L.n; i += gs) {
      if (masked(L.mask, i)) continue;
      const T xo = ldc(cur + i);  // ahead of the prolongation's loads
      cur[i] = T(1) * coarse_prol<T, DIM>(L, C, sol[l + 1], i) + xo;
    }
    cl.sync();
    T* s0 = cur;
    double dn = 0.0;
    for (int it = 0; it < nu; ++it) {
      double acc = 0.0;
      const double dv = sqrt(dn);
      const bool skip = it > 0 && (!isfinite(dv) || dv <= double(eps_of<T>()) * double(eps_of<T>()));
      for (uint32_t i = gt; i < L.n; i += gs) {
        const RowIn<T> in = row_in(L, cur, b, i);  // ahead of the row's gathers
        const T o0 = skip ? ldc(s0 + i) : T(0);
        const T s = coarse_row<T, DIM>(L, cur, int32_t(i));
        oth[i] = post_row(om, in, o0, s, skip, it == 0, acc);
      }
      if (it == 0) {
        dn = cluster_sum<THREADS>(acc, part[rk++ & 1], sh, cl);
        if (gt == 0) *L.dn = dn;
        if (nu == 1) {
          // the smoother skipped: its result is the prolongated iterate (k_skip_fix)
          const double d1 = sqrt(dn);
          if (!isfinite(d1) || d1 <= double(eps_of<T>()) * double(eps_of<T>())) {
            for (uint32_t i = gt; i < L.n; i += gs) oth[i] = ldc(s0 + i);
            cl.sync();
          }
        }
      } else {
        cl.sync();
      }
      T* tmp = cur; cur = oth; oth = tmp;
    }
    sol[l] = cur;
  }
}

}  // namespace fb
