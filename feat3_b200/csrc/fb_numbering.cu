// FEAT3's DOF and cell numbering of the refined unit square / cube, computed on the device.
//
// FEAT3 builds a structured hierarchy by refining the unit cube (UnitCubeFactory,
// kernel/geometry/common_factories.hpp:71-235) with the standard refinery
// (conformal_mesh.hpp:439-528). Its numbering follows from three rules:
//  * the vertices of a refined mesh are the old vertices, then one new vertex per edge, quad
//    and hexa, in entity order (intern/standard_vertex_refiner.hpp:65-110, 195-253);
//  * the edges (quads, hexas) of a refined mesh are the children of the edges, then of the quads,
//    then of the hexas, each parent's children consecutive (intern/standard_index_refiner.hpp:
//    2762-2840), ordered and oriented as StandardIndexRefiner<Hypercube<d>,c,0> lists their
//    vertices (:1346-1402, 1414-1602, 1723-2174);
//  * Lagrange DOFs are numbered vertices first, then edges, quads, hexas
//    (space/dof_mapping_common.hpp:255-330), so the Q2 numbering on level L is the vertex
//    numbering on level L+1.
// Starting from the unit cube, whose vertex i sits at the bits of i and whose edges and faces
// follow FaceIndexMapping (intern/face_index_mapping.hpp:119-183), every entity the refinement
// creates has its local axes along increasing global axes, in positive direction (each child
// keeps its parent's frame, and the interior edges and quads of a parent run from its lower to
// its upper side). So the FEAT index of a lattice point follows from a descent through the
// levels: the smallest entity containing the point on each level, its index from its parent's
// index and the child's position in the parent. One thread per point, O(level) integer work,
// no mesh stored. The CPU oracle restates the refinement itself (entity by entity) and is
// pinned to the reference's own numbering; the tests compare the two.
#include "fb_mg_internal.cuh"

namespace fb {
namespace {

struct Counts { uint64_t V, E, Q; };

// entity counts of the level with n cells per side
__device__ __forceinline__ Counts level_counts(int D, uint64_t n) {
  const uint64_t m = n + 1;
  if (D == 2) return {m * m, 2 * n * m, n * n};
  return {m * m * m, 3 * n * m * m, 3 * n * n * m};
}

// FEAT index of lattice point p (coordinates 0..2^lv) in the vertex numbering of level lv
template <int D>
__device__ uint64_t feat_vertex(const uint32_t* p, int lv) {
  uint32_t s = 1u << lv;  // spacing of the current level in lattice units
  // level 0: the unit cube's vertex, edge, face or the cell holding p
  unsigned span = 0;
  uint32_t k[3] = {0, 0, 0};
  for (int a = 0; a < D; ++a) {
    if (p[a] == 0 || p[a] == s) k[a] = p[a] ? 1 : 0;
    else span |= 1u << a;
  }
  int d = __popc(span);
  uint64_t idx;
  if (d == 0) {
    idx = 0;
    for (int a = 0; a < D; ++a) idx |= uint64_t(k[a]) << a;
    return idx;
  }
  if (d == D) {
    idx = 0;
  } else if (D == 2) {  // edges {0,1},{2,3} along x, {0,2},{1,3} along y
    idx = (span & 1) ? k[1] : 2 + k[0];
  } else if (d == 1) {  // edges along x (0..3), y (4..7), z (8..11)
    if (span & 1) idx = k[1] + 2 * k[2];
    else if (span & 2) idx = 4 + k[0] + 2 * k[2];
    else idx = 8 + k[0] + 2 * k[1];
  } else {              // faces normal to z (0,1), y (2,3), x (4,5)
    if (!(span & 4)) idx = k[2];
    else if (!(span & 2)) idx = 2 + k[1];
    else idx = 4 + k[0];
  }
  for (int l = 1; l <= lv; ++l) {
    const uint32_t h = s >> 1;
    const Counts c = level_counts(D, uint64_t(1) << (l - 1));
    // position of p in the current entity, per local axis (the spanning axes in increasing order)
    unsigned nspan = 0, half = 0, mid = 0;
    int b = 0;
    for (int a = 0; a < D; ++a) {
      if (!(span & (1u << a))) continue;
      const uint32_t r = p[a] & (s - 1);
      if (r == h) mid |= 1u << b;
      else {
        nspan |= 1u << a;
        if (r > h) half |= 1u << b;
      }
      ++b;
    }
    const int nd = __popc(nspan);
    if (nd == 0)  // p is the entity's centre: a new vertex of this level, index fixed from here on
      return c.V + (d == 1 ? 0 : d == 2 ? c.E : c.E + c.Q) + idx;
    if (nd == d) {
      idx = (idx << d) + half;  // children of the same dimension, in local tensor order
    } else if (nd == 1) {
      const int br = __ffs(~mid & ((1u << d) - 1)) - 1;  // the local axis the child edge runs along
      const unsigned hb = (half >> br) & 1u;
      if (d == 2) idx = 2 * c.E + 4 * idx + (br == 1 ? hb : 2 + hb);
      else idx = 2 * c.E + 4 * c.Q + 6 * idx + 2 * (2 - br) + hb;
    } else {  // an interior quad of a hexa, normal to local axis `nl`
      const int nl = __ffs(mid) - 1;
      const unsigned h0 = half & 1u, h1 = (half >> 1) & 1u, h2 = (half >> 2) & 1u;
      const unsigned j = nl == 0 ? h1 + 2 * h2 : nl == 1 ? 4 + h0 + 2 * h2 : 8 + h0 + 2 * h1;
      idx = 4 * c.Q + 12 * idx + j;
    }
    span = nspan;
    d = nd;
    s = h;
  }
  return idx;  // not reached for points of the level-lv lattice
}

template <int D>
__global__ void k_feat_dofs(int lv, uint32_t M1, uint64_t total, uint32_t* dof_lex) {
  for (uint64_t t = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; t < total; t += uint64_t(gridDim.x) * blockDim.x) {
    uint32_t p[3];
    uint64_t r = t;
    for (int a = 0; a < D; ++a) { p[a] = uint32_t(r % M1); r /= M1; }
    dof_lex[feat_vertex<D>(p, lv)] = uint32_t(t);
  }
}

// FEAT cell index = the children indices of the descent, D bits per level (child j of a hexa
// sits at the octant of its parent's vertex j)
template <int D>
__global__ void k_feat_cells(int lv, uint64_t total, uint32_t* cell_lex) {
  const uint32_t N = 1u << lv;
  for (uint64_t t = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; t < total; t += uint64_t(gridDim.x) * blockDim.x) {
    uint32_t c[3];
    uint64_t r = t;
    for (int a = 0; a < D; ++a) { c[a] = uint32_t(r % N); r /= N; }
    uint64_t idx = 0;
    for (int l = lv - 1; l >= 0; --l) {
      unsigned j = 0;
      for (int a = 0; a < D; ++a) j |= ((c[a] >> l) & 1u) << a;
      idx = (idx << D) | j;
    }
    cell_lex[idx] = uint32_t(t);
  }
}

__global__ void k_perm_to(double* __restrict__ dst, const double* __restrict__ src, const uint32_t* __restrict__ perm,
                          uint64_t n) {
  for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x)
    dst[perm[i]] = src[i];
}

__global__ void k_perm_from(double* __restrict__ dst, const double* __restrict__ src, const uint32_t* __restrict__ perm,
                            uint64_t n) {
  for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x)
    dst[i] = __ldg(src + perm[i]);
}

}  // namespace

int perm_to_lattice(fb_mg* m, double* dst, const double* src, const uint32_t* perm, uint64_t n) {
  k_perm_to<<<ew_grid(n), 256, 0, m->stream>>>(dst, src, perm, n);
  m->launches++;
  return cudaGetLastError() == cudaSuccess ? FB_OK : FB_ERR_CUDA;
}

int perm_from_lattice(fb_mg* m, double* dst, const double* src, const uint32_t* perm, uint64_t n) {
  k_perm_from<<<ew_grid(n), 256, 0, m->stream>>>(dst, src, perm, n);
  m->launches++;
  return cudaGetLastError() == cudaSuccess ? FB_OK : FB_ERR_CUDA;
}

int in_lattice(fb_mg* m, const double* src, double* stage, const double** out) {
  *out = src;
  if (!m->feat_dof) return FB_OK;
  *out = stage;
  return perm_to_lattice(m, stage, src, m->feat_dof, m->L[0].n);
}

int feat_numbering(int dim, int degree, int level, uint32_t* dof_lex, uint32_t* cell_lex, cudaStream_t s) {
  if ((dim != 2 && dim != 3) || (degree != 1 && degree != 2) || level < 0) return FB_ERR_INVALID;
  const int lv = level + (degree == 2 ? 1 : 0);
  const uint64_t M1 = (uint64_t(1) << lv) + 1;
  const uint64_t ndof = dim == 2 ? M1 * M1 : M1 * M1 * M1;
  const uint64_t ncell = uint64_t(1) << (dim * level);
  if (lv > (dim == 2 ? 15 : 10) || ndof > 0xffffffffull) return FB_ERR_TOO_LARGE;
  const int threads = 256;
  auto grid = [&](uint64_t n) { return unsigned(std::min<uint64_t>((n + threads - 1) / threads, 148ull * 64)); };
  if (dof_lex) {
    if (dim == 2) k_feat_dofs<2><<<grid(ndof), threads, 0, s>>>(lv, uint32_t(M1), ndof, dof_lex);
    else k_feat_dofs<3><<<grid(ndof), threads, 0, s>>>(lv, uint32_t(M1), ndof, dof_lex);
    if (cudaGetLastError() != cudaSuccess) return FB_ERR_CUDA;
  }
  if (cell_lex) {
    if (dim == 2) k_feat_cells<2><<<grid(ncell), threads, 0, s>>>(level, ncell, cell_lex);
    else k_feat_cells<3><<<grid(ncell), threads, 0, s>>>(level, ncell, cell_lex);
    if (cudaGetLastError() != cudaSuccess) return FB_ERR_CUDA;
  }
  return FB_OK;
}

}  // namespace fb

extern "C" int fb_feat_numbering(int dim, int degree, int level, uint32_t* dof_lex, uint32_t* cell_lex,
                                 fb_stream_t stream) {
  return fb::feat_numbering(dim, degree, level, dof_lex, cell_lex, static_cast<cudaStream_t>(stream));
}
