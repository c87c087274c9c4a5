// Structured Q1/Q2 hierarchies assembled on the device.
//
// Mesh: the unit square/cube refined `level` times (N = 2^level cells per side); degrees
// of freedom on the lexicographic lattice of (degree*N + 1)^dim points. The element
// stiffness of a cube of side h with a constant coefficient k_e is k_e (h/2)^(dim-2) K_ref,
// K_ref integrated on [-1,1]^dim with 3-point Gauss-Legendre per direction -- the rule the
// reference selects for "auto-degree:5" (kernel/cubature/auto_alias.hpp) and which is exact
// for these integrands (kernel/assembly/bilinear_operator_assembler.hpp:218-339,
// common_operators.hpp:36-97).
//
// Instead of the reference's per-cell scatter into a CSR pattern, every row gathers its
// entries from the (at most 2^dim) cells around it. Cells are visited in ascending
// index order, which is the order in which the cell-wise scatter adds into an entry, so
// the FP64 values are the same numbers the cell-wise assembly produces. The rows are
// written straight into the SELL-C (C = 32) slots of the level matrix.
//
// Transfers: the Q1/Q2 spaces of two consecutive levels are nested, so the L2 projection
// of kernel/assembly/grid_transfer.hpp:304-321 reduces to interpolation; P is the
// Kronecker product of 1D interpolation matrices and R = P^T the product of their
// transposes (tutorial_05_multigrid.cpp:302).
#include "fb_mg_internal.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#undef FB_CHECK_LAUNCH
#define FB_CHECK_LAUNCH()                                                              \
  do {                                                                                 \
    cudaError_t _e = cudaGetLastError();                                               \
    if (_e == cudaSuccess && fb::debug_enabled()) _e = fb::debug_sync(m->stream, __FILE__, __LINE__); \
    if (_e != cudaSuccess) return FB_ERR_CUDA;                                         \
  } while (0)

namespace fb {

struct Geom {
  int dim, p;      // dimension, polynomial degree
  uint32_t N;      // cells per side
  uint32_t M;      // lattice intervals per side (p*N)
  uint32_t M1;     // lattice points per side
};

__host__ __device__ inline void lat_coords(uint64_t i, const Geom& g, uint32_t c[3]) {
  c[0] = uint32_t(i % g.M1);
  c[1] = uint32_t((i / g.M1) % g.M1);
  c[2] = g.dim == 3 ? uint32_t(i / (uint64_t(g.M1) * g.M1)) : 0u;
}

// lattice range of the columns coupled to coordinate X (union of its cells)
__host__ __device__ inline void col_range(uint32_t X, const Geom& g, uint32_t& lo, uint32_t& hi) {
  if (g.p == 1 || (X & 1u) == 0u) {
    const uint32_t w = uint32_t(g.p);
    lo = X >= w ? X - w : 0u;
    hi = X + w <= g.M ? X + w : g.M;
  } else {
    lo = X - 1u;
    hi = X + 1u;
  }
}

// cells (1D indices, ascending) containing lattice coordinate X
__host__ __device__ inline int cells_of(uint32_t X, const Geom& g, uint32_t e[2]) {
  if (g.p == 2 && (X & 1u)) { e[0] = (X - 1u) / 2u; return 1; }
  const uint32_t v = g.p == 1 ? X : X / 2u;  // vertex index along this direction
  int k = 0;
  if (v > 0) e[k++] = v - 1u;
  if (v < g.N) e[k++] = v;
  return k;
}

__host__ __device__ inline uint32_t row_length(uint64_t row, const Geom& g) {
  uint32_t c[3];
  lat_coords(row, g, c);
  uint32_t len = 1;
  for (int d = 0; d < g.dim; ++d) {
    uint32_t lo, hi;
    col_range(c[d], g, lo, hi);
    len *= hi - lo + 1u;
  }
  return len;
}

// visits the entries of `row` in ascending column order: emit(j, col, value)
template<typename F>
__host__ __device__ inline void row_entries(uint64_t row, const Geom& g, const double* k, const double* kref,
                                            double sc, F&& emit) {
  uint32_t c[3];
  lat_coords(row, g, c);
  uint32_t lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0}, ce[3][2] = {{0, 0}, {0, 0}, {0, 0}};
  int nce[3] = {1, 1, 1};
  for (int d = 0; d < g.dim; ++d) {
    col_range(c[d], g, lo[d], hi[d]);
    nce[d] = cells_of(c[d], g, ce[d]);
  }
  const int q1 = g.p + 1;
  const int nloc = g.dim == 2 ? q1 * q1 : q1 * q1 * q1;
  const uint64_t M1 = g.M1;
  uint32_t j = 0;
  for (uint32_t z = lo[2]; z <= hi[2]; ++z)
    for (uint32_t y = lo[1]; y <= hi[1]; ++y)
      for (uint32_t x = lo[0]; x <= hi[0]; ++x) {
        const uint32_t cc[3] = {x, y, z};
        double v = 0.0;
        for (int ez = 0; ez < nce[2]; ++ez)
          for (int ey = 0; ey < nce[1]; ++ey)
            for (int ex = 0; ex < nce[0]; ++ex) {
              const uint32_t e3[3] = {ce[0][ex], ce[1][ey], ce[2][ez]};
              int a = 0, b = 0, mul = 1;
              bool inside = true;
              for (int d = 0; d < g.dim; ++d) {
                const int base = int(e3[d]) * g.p;
                const int lr = int(c[d]) - base, lc = int(cc[d]) - base;
                if (lc < 0 || lc > g.p) { inside = false; break; }
                a += lr * mul; b += lc * mul; mul *= q1;
              }
              if (!inside) continue;
              const uint64_t eidx = uint64_t(e3[0]) + uint64_t(g.N) * (uint64_t(e3[1]) + uint64_t(g.N) * e3[2]);
              const double ke = k ? k[eidx] : 1.0;
              // separate multiply and add roundings (no contraction), as in a cell-wise scatter
#ifdef __CUDA_ARCH__
              v = __dadd_rn(v, __dmul_rn(__dmul_rn(ke, sc), kref[a * nloc + b]));
#else
              v += ke * sc * kref[a * nloc + b];
#endif
            }
        emit(j++, uint32_t(uint64_t(x) + M1 * (uint64_t(y) + M1 * z)), v);
      }
}

__global__ void k_rowlen(Geom g, uint64_t n, uint32_t* rl, uint32_t* cl) {
  const uint64_t row = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x;
  uint32_t len = row < n ? row_length(row, g) : 0u;
  if (row < n) rl[row] = len;
  const uint32_t mx = __reduce_max_sync(0xffffffffu, len);
  if ((threadIdx.x & 31) == 0 && row < n) cl[row >> 5] = mx;
}

// one thread per SELL slot row (nchunks*32 threads): rows beyond n in the last chunk get
// padding too, because the SELL kernels load every lane's column and gather x with it
__global__ void k_fill_sell(Geom g, uint64_t n, uint32_t nchunks, const uint32_t* __restrict__ cs,
                            const uint32_t* __restrict__ cl, const double* __restrict__ k,
                            const double* __restrict__ kref, double sc, uint32_t* col, double* val) {
  const uint64_t row = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x;
  if (row >= uint64_t(nchunks) * 32) return;
  const uint32_t ch = uint32_t(row >> 5), t = uint32_t(row & 31);
  const uint64_t base = uint64_t(cs[ch]) + t;
  uint32_t used = 0;
  if (row < n) {
    row_entries(row, g, k, kref, sc, [&](uint32_t j, uint32_t c, double v) {
      col[base + uint64_t(j) * 32] = c;
      val[base + uint64_t(j) * 32] = v;
      used = j + 1;
    });
  }
  const uint32_t pad_col = row < n ? uint32_t(row) : uint32_t(n - 1);
  for (uint32_t j = used; j < cl[ch]; ++j) {
    col[base + uint64_t(j) * 32] = pad_col;
    val[base + uint64_t(j) * 32] = 0.0;
  }
}

// implicit-column (stencil) copy of a Q1 level matrix: slot j of row r holds a(r, r + off[j])
__global__ void k_fill_stencil(Geom g, uint64_t n, const double* __restrict__ k, const double* __restrict__ kref,
                               double sc, double* val) {
  const uint64_t row = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x;
  if (row >= n) return;
  const int S = g.dim == 3 ? 27 : 9;
  const uint64_t c = row >> 5, t = row & 31;
  uint32_t rc[3];
  lat_coords(row, g, rc);
  row_entries(row, g, k, kref, sc, [&](uint32_t, uint32_t col, double v) {
    uint32_t cc[3];
    lat_coords(col, g, cc);
    int slot = 0;
    for (int d = g.dim - 1; d >= 0; --d) slot = slot * 3 + (int(cc[d]) - int(rc[d]) + 1);
    val[(c * S + slot) * 32 + t] = v;
  });
}

__global__ void k_mask(Geom g, uint64_t n, uint32_t* mask) {
  const uint64_t w = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x;
  if (w * 32 >= n) return;
  uint32_t bits = 0;
  for (int b = 0; b < 32; ++b) {
    const uint64_t i = w * 32 + b;
    if (i >= n) break;
    uint32_t c[3];
    lat_coords(i, g, c);
    bool bd = false;
    for (int d = 0; d < g.dim; ++d) bd = bd || c[d] == 0 || c[d] == g.M;
    if (bd) bits |= 1u << b;
  }
  mask[w] = bits;
}

__global__ void k_to_f32(float* dst, const double* __restrict__ src, uint64_t n) {
  const uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x;
  if (i < n) dst[i] = float(src[i]);
}

// coarse coefficient = mean of the 2^dim children
__global__ void k_coarsen_k(int dim, uint32_t Nc, const double* __restrict__ kf, double* kc) {
  uint64_t nec = uint64_t(Nc) * Nc * (dim == 3 ? Nc : 1);
  const uint64_t e = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x;
  if (e >= nec) return;
  const uint64_t Nf = 2ull * Nc;
  const uint64_t cx = e % Nc, cy = (e / Nc) % Nc, cz = dim == 3 ? e / (uint64_t(Nc) * Nc) : 0;
  double s = 0.0;
  for (int c = 0; c < (1 << dim); ++c) {
    const uint64_t fx = 2 * cx + (c & 1), fy = 2 * cy + ((c >> 1) & 1), fz = dim == 3 ? 2 * cz + ((c >> 2) & 1) : 0;
    s += kf[fx + Nf * (fy + Nf * fz)];
  }
  kc[e] = s / double(1 << dim);
}

// Kronecker product of a 1D CSR matrix with itself (dim times), lexicographic ordering
struct Kron1D {
  uint32_t rows, cols;          // 1D sizes
  const uint32_t* rp;           // rows+1
  const uint32_t* ci;
  const double* va;
  uint64_t total;               // nnz of the 1D matrix
};
__global__ void k_kron(int dim, Kron1D a, uint32_t* rp, uint32_t* col, double* val) {
  const uint64_t nrows = uint64_t(a.rows) * a.rows * (dim == 3 ? a.rows : 1);
  const uint64_t row = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x;
  if (row > nrows) return;
  if (row == nrows) {
    rp[nrows] = uint32_t(a.total * a.total * (dim == 3 ? a.total : 1));
    return;
  }
  const uint32_t X = uint32_t(row % a.rows), Y = uint32_t((row / a.rows) % a.rows), Z = dim == 3 ? uint32_t(row / (uint64_t(a.rows) * a.rows)) : 0u;
  const uint64_t S = a.total;
  const uint64_t lx = a.rp[X + 1] - a.rp[X], ly = a.rp[Y + 1] - a.rp[Y];
  uint64_t start;
  if (dim == 3) {
    const uint64_t lz = a.rp[Z + 1] - a.rp[Z];
    start = uint64_t(a.rp[Z]) * S * S + lz * (uint64_t(a.rp[Y]) * S + ly * a.rp[X]);
  } else {
    start = uint64_t(a.rp[Y]) * S + ly * a.rp[X];
  }
  (void)lx;
  rp[row] = uint32_t(start);
  uint64_t k = start;
  const uint64_t C = a.cols;
  const uint32_t zb = dim == 3 ? a.rp[Z] : 0u, ze = dim == 3 ? a.rp[Z + 1] : 1u;
  for (uint32_t iz = zb; iz < ze; ++iz) {
    const double wz = dim == 3 ? a.va[iz] : 1.0;
    const uint64_t cz = dim == 3 ? a.ci[iz] : 0u;
    for (uint32_t iy = a.rp[Y]; iy < a.rp[Y + 1]; ++iy)
      for (uint32_t ix = a.rp[X]; ix < a.rp[X + 1]; ++ix) {
        col[k] = uint32_t(a.ci[ix] + C * (a.ci[iy] + C * cz));
        val[k] = a.va[ix] * a.va[iy] * wz;
        ++k;
      }
  }
}

// ---- load vectors (common_functionals.hpp:137-225 with the analytic functions of
//      kernel/analytic/common.hpp), gathered per row over the cells around the dof
__device__ inline double ebs(double x) {
  return (exp(-(2.0 * x - 1.0) * (2.0 * x - 1.0)) - exp(-1.0)) / (1.0 - exp(-1.0));
}
__device__ inline double ebs_xx(double x) {
  return (64.0 * x * (1.0 - x) - 8.0) * exp(-(2.0 * x - 1.0) * (2.0 * x - 1.0)) / (exp(-1.0) - 1.0);
}
__host__ __device__ inline void basis1d(int p, double t, double* v) {
  if (p == 1) { v[0] = 0.5 * (1.0 - t); v[1] = 0.5 * (1.0 + t); }
  else { v[0] = 0.5 * t * (t - 1.0); v[1] = 1.0 - t * t; v[2] = 0.5 * t * (t + 1.0); }
}
__global__ void k_rhs(Geom g, uint64_t n, int kind, const uint32_t* mask, double* rhs) {
  const uint64_t row = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x;
  if (row >= n) return;
  if (masked(mask, uint32_t(row))) { rhs[row] = 0.0; return; }
  const double gx[3] = {-sqrt(3.0 / 5.0), 0.0, sqrt(3.0 / 5.0)};
  const double gw[3] = {5.0 / 9.0, 8.0 / 9.0, 5.0 / 9.0};
  const double h = 1.0 / double(g.N);
  const double det = pow(0.5 * h, double(g.dim));
  const double pi = 3.14159265358979323846;
  uint32_t c[3];
  lat_coords(row, g, c);
  uint32_t ce[3][2] = {{0, 0}, {0, 0}, {0, 0}};
  int nce[3] = {1, 1, 1};
  for (int d = 0; d < g.dim; ++d) nce[d] = cells_of(c[d], g, ce[d]);
  double acc = 0.0;
  const int nq = g.dim == 2 ? 9 : 27;
  for (int ez = 0; ez < nce[2]; ++ez)
    for (int ey = 0; ey < nce[1]; ++ey)
      for (int ex = 0; ex < nce[0]; ++ex) {
        const uint32_t e3[3] = {ce[0][ex], ce[1][ey], ce[2][ez]};
        double cell = 0.0;
        for (int q = 0; q < nq; ++q) {
          const int qi[3] = {q % 3, (q / 3) % 3, q / 9};
          double w = det, xq[3] = {0, 0, 0}, phi = 1.0;
          for (int d = 0; d < g.dim; ++d) {
            w *= gw[qi[d]];
            xq[d] = (double(e3[d]) + 0.5 * (gx[qi[d]] + 1.0)) * h;
            double bv[3];
            basis1d(g.p, gx[qi[d]], bv);
            phi *= bv[int(c[d]) - int(e3[d]) * g.p];
          }
          double f;
          if (kind == 0) {
            f = double(g.dim) * pi * pi;
            for (int d = 0; d < g.dim; ++d) f *= sin(pi * xq[d]);
          } else if (kind == 1) {
            f = 1.0;
          } else {
            f = 0.0;
            for (int a = 0; a < g.dim; ++a) {
              double t = ebs_xx(xq[a]);
              for (int b = 0; b < g.dim; ++b) if (b != a) t *= ebs(xq[b]);
              f -= t;
            }
          }
          cell += w * f * phi;
        }
        acc += cell;
      }
  rhs[row] = acc;
}

// dJ/dk_e = -lambda_e^T K_e^(1) u_e on the finest level
__global__ void k_elem_grad(Geom g, uint64_t ne, const double* __restrict__ u, const double* __restrict__ lam,
                            const double* __restrict__ kref, double sc, double* grad) {
  const uint64_t e = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x;
  if (e >= ne) return;
  const uint64_t ex = e % g.N, ey = (e / g.N) % g.N, ez = g.dim == 3 ? e / (uint64_t(g.N) * g.N) : 0;
  const int q1 = g.p + 1;
  const int nloc = g.dim == 2 ? q1 * q1 : q1 * q1 * q1;
  double ul[27], ll[27];
  for (int a = 0; a < nloc; ++a) {
    const int ax = a % q1, ay = (a / q1) % q1, az = a / (q1 * q1);
    const uint64_t X = ex * g.p + ax, Y = ey * g.p + ay, Z = ez * g.p + az;
    const uint64_t i = X + uint64_t(g.M1) * (Y + uint64_t(g.M1) * Z);
    ul[a] = u[i];
    ll[a] = lam[i];
  }
  double s = 0.0;
  for (int a = 0; a < nloc; ++a) {
    double ka = 0.0;
    for (int b = 0; b < nloc; ++b) ka += kref[a * nloc + b] * ul[b];
    s += ll[a] * ka;
  }
  grad[e] = -sc * s;
}

__global__ void k_adj_rhs(double* g, const double* __restrict__ u, const double* __restrict__ t, const uint32_t* mask, uint32_t n) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    g[i] = masked(mask, i) ? 0.0 : u[i] - t[i];
}

// ---------------------------------------------------------------------------------------
// host helpers
static void build_kref(int dim, int p, std::vector<double>& K, int& nloc) {
  const int q1 = p + 1;
  nloc = dim == 2 ? q1 * q1 : q1 * q1 * q1;
  K.assign(size_t(nloc) * nloc, 0.0);
  const double a = std::sqrt(3.0 / 5.0);
  const double gx[3] = {-a, 0.0, a}, gw[3] = {5.0 / 9.0, 8.0 / 9.0, 5.0 / 9.0};
  const int nq = dim == 2 ? 9 : 27;
  std::vector<double> grad(size_t(nloc) * dim);
  for (int q = 0; q < nq; ++q) {
    const int qi[3] = {q % 3, (q / 3) % 3, q / 9};
    double w = 1.0, v[3][3], dv[3][3];
    for (int d = 0; d < dim; ++d) {
      w *= gw[qi[d]];
      const double t = gx[qi[d]];
      if (p == 1) { v[d][0] = 0.5 * (1.0 - t); v[d][1] = 0.5 * (1.0 + t); dv[d][0] = -0.5; dv[d][1] = 0.5; }
      else {
        v[d][0] = 0.5 * t * (t - 1.0); v[d][1] = 1.0 - t * t; v[d][2] = 0.5 * t * (t + 1.0);
        dv[d][0] = t - 0.5; dv[d][1] = -2.0 * t; dv[d][2] = t + 0.5;
      }
    }
    for (int i = 0; i < nloc; ++i) {
      const int li[3] = {i % q1, (i / q1) % q1, i / (q1 * q1)};
      for (int c = 0; c < dim; ++c) {
        double gg = 1.0;
        for (int d = 0; d < dim; ++d) gg *= (d == c) ? dv[d][li[d]] : v[d][li[d]];
        grad[size_t(i) * dim + c] = gg;
      }
    }
    for (int i = 0; i < nloc; ++i)
      for (int j = 0; j < nloc; ++j) {
        double s = 0.0;
        for (int c = 0; c < dim; ++c) s += grad[size_t(j) * dim + c] * grad[size_t(i) * dim + c];
        K[size_t(i) * nloc + j] += w * s;
      }
  }
}

// levels of at least this many rows build their assembled copies on first use
constexpr uint32_t kLazyRows = 1u << 20;

static double elem_scale(int dim, int level) {
  const double h = 1.0 / double(1u << level);
  return std::pow(0.5 * h, double(dim - 2));
}

// 1D interpolation from Mc intervals (coarse) onto Mf = 2 Mc (fine), CSR over fine points
static void prol1d(int p, uint32_t Mf, std::vector<uint32_t>& rp, std::vector<uint32_t>& ci, std::vector<double>& va) {
  rp.assign(Mf + 2, 0); ci.clear(); va.clear();
  for (uint32_t f = 0; f <= Mf; ++f) {
    if (p == 1) {
      if (f % 2 == 0) { ci.push_back(f / 2); va.push_back(1.0); }
      else { ci.push_back(f / 2); va.push_back(0.5); ci.push_back(f / 2 + 1); va.push_back(0.5); }
    } else {
      const uint32_t c = std::min<uint32_t>(f / 4, Mf / 4 - 1);
      const int off = int(f - 4 * c);
      const double t = -1.0 + 0.5 * off;
      double v[3];
      basis1d(2, t, v);
      for (int a = 0; a < 3; ++a)
        if (v[a] != 0.0) { ci.push_back(2 * c + a); va.push_back(v[a]); }
    }
    rp[f + 1] = uint32_t(ci.size());
  }
}

static void transpose1d(uint32_t rows, uint32_t cols, const std::vector<uint32_t>& rp, const std::vector<uint32_t>& ci,
                        const std::vector<double>& va, std::vector<uint32_t>& trp, std::vector<uint32_t>& tci,
                        std::vector<double>& tva) {
  trp.assign(cols + 1, 0);
  for (auto c : ci) trp[c + 1]++;
  for (uint32_t i = 0; i < cols; ++i) trp[i + 1] += trp[i];
  tci.resize(ci.size()); tva.resize(va.size());
  std::vector<uint32_t> pos(trp.begin(), trp.end() - 1);
  for (uint32_t r = 0; r < rows; ++r)
    for (uint32_t k = rp[r]; k < rp[r + 1]; ++k) { tci[pos[ci[k]]] = r; tva[pos[ci[k]]] = va[k]; pos[ci[k]]++; }
}

static int build_kron(fb_mg* m, DevCsr& D, int dim, uint32_t rows1, uint32_t cols1, const std::vector<uint32_t>& rp,
                      const std::vector<uint32_t>& ci, const std::vector<double>& va) {
  uint32_t *drp = nullptr, *dci = nullptr;
  double* dva = nullptr;
  FB_TRY(dupload(m, &drp, rp.data(), rp.size()));
  FB_TRY(dupload(m, &dci, ci.data(), ci.size()));
  FB_TRY(dupload(m, &dva, va.data(), va.size()));
  Kron1D a{rows1, cols1, drp, dci, dva, uint64_t(ci.size())};
  const uint64_t nrows = uint64_t(rows1) * rows1 * (dim == 3 ? rows1 : 1);
  const uint64_t nnz = a.total * a.total * (dim == 3 ? a.total : 1);
  if (nrows > 0xffffffffull || nnz > 0xffffffffull) return FB_ERR_INVALID;
  D.rows = uint32_t(nrows);
  D.cols = uint32_t(uint64_t(cols1) * cols1 * (dim == 3 ? cols1 : 1));
  D.nnz = nnz;
  FB_TRY(dalloc(m, &D.rp, nrows + 1));
  FB_TRY(dalloc(m, &D.col, nnz));
  FB_TRY(dalloc(m, &D.v64, nnz));
  k_kron<<<grid_for(nrows + 1, 256), 256, 0, m->stream>>>(dim, a, D.rp, D.col, D.v64);
  FB_CHECK_LAUNCH();
  return FB_OK;
}

// the level's structure without its values: SELL / stencil shapes, the true nonzero count, the
// stencil offsets and the Dirichlet mask (the lattice boundary)
static int build_level_meta(fb_mg* m, Level& L, const Geom& g) {
  const uint64_t n = L.n;
  DevSell& S = L.A;
  S.rows = S.cols = uint32_t(n);
  S.nchunks = uint32_t((n + 31) / 32);
  // true nonzeros: sum of row lengths (closed form per direction)
  uint64_t nnz1 = 0;
  for (uint32_t X = 0; X <= g.M; ++X) {
    uint32_t lo, hi;
    col_range(X, g, lo, hi);
    nnz1 += hi - lo + 1;
  }
  S.nnz = nnz1 * nnz1 * (g.dim == 3 ? nnz1 : 1);
  if (g.p == 1) {
    DevStencil& St = L.St;
    St.S = g.dim == 3 ? 27 : 9;
    St.nchunks = S.nchunks;
    int j = 0;
    const int z0 = g.dim == 3 ? -1 : 0, z1 = g.dim == 3 ? 1 : 0;
    for (int dz = z0; dz <= z1; ++dz)
      for (int dy = -1; dy <= 1; ++dy)
        for (int dx = -1; dx <= 1; ++dx)
          St.off[j++] = int32_t((int64_t(dz) * g.M1 + dy) * g.M1 + dx);
  }
  FB_TRY(dalloc(m, &L.mask, (n + 31) / 32));
  k_mask<<<grid_for((n + 31) / 32, 256), 256, 0, m->stream>>>(g, n, L.mask);
  FB_CHECK_LAUNCH();
  L.mask_boundary = true;
  return FB_OK;
}

// the level's assembled values: SELL (row lengths, chunk starts, columns, FP64 values) and, for Q1,
// the implicit-column stencil copy (all rows padded to the full 3^dim stencil; absent neighbours = 0)
static int build_level_values(fb_mg* m, Level& L, const Geom& g, double sc) {
  const uint64_t n = L.n;
  DevSell& S = L.A;
  FB_TRY(dalloc(m, &S.rl, n));
  FB_TRY(dalloc(m, &S.cl, S.nchunks));
  FB_TRY(dalloc(m, &S.cs, S.nchunks + 1));
  k_rowlen<<<grid_for(uint64_t(S.nchunks) * 32, 256), 256, 0, m->stream>>>(g, n, S.rl, S.cl);
  FB_CHECK_LAUNCH();
  std::vector<uint32_t> cl(S.nchunks), cs(S.nchunks + 1, 0);
  FB_CUDA(cudaMemcpyAsync(cl.data(), S.cl, sizeof(uint32_t) * S.nchunks, cudaMemcpyDeviceToHost, m->stream));
  FB_CUDA(cudaStreamSynchronize(m->stream));
  uint64_t acc = 0;
  for (uint32_t c = 0; c < S.nchunks; ++c) {
    cs[c] = uint32_t(acc);
    acc += uint64_t(cl[c]) * 32;
    if (acc > 0xffffffffull) return FB_ERR_INVALID;
  }
  cs[S.nchunks] = uint32_t(acc);
  S.nent = acc;
  FB_CUDA(cudaMemcpyAsync(S.cs, cs.data(), sizeof(uint32_t) * cs.size(), cudaMemcpyHostToDevice, m->stream));
  FB_CUDA(cudaStreamSynchronize(m->stream));
  FB_TRY(dalloc(m, &S.col, S.nent));
  FB_TRY(dalloc(m, &S.v64, S.nent));
  k_fill_sell<<<grid_for(uint64_t(S.nchunks) * 32, 128), 128, 0, m->stream>>>(g, n, S.nchunks, S.cs, S.cl, L.k, m->kref,
                                                                             sc, S.col, S.v64);
  FB_CHECK_LAUNCH();
  if (g.p == 1) {
    DevStencil& St = L.St;
    const uint64_t ns = uint64_t(St.nchunks) * St.S * 32;
    FB_TRY(dalloc(m, &St.v64, ns));
    FB_CUDA(cudaMemsetAsync(St.v64, 0, sizeof(double) * ns, m->stream));
    k_fill_stencil<<<grid_for(n, 128), 128, 0, m->stream>>>(g, n, L.k, m->kref, sc, St.v64);
    FB_CHECK_LAUNCH();
  }
  return FB_OK;
}

static int build_level(fb_mg* m, Level& L, const Geom& g, double sc) {
  FB_TRY(build_level_meta(m, L, g));
  return build_level_values(m, L, g, sc);
}

// diagonal of the level matrix from the row gather that fills the SELL (bit-identical to its
// stored diagonal entry), without the assembled matrix
__global__ void k_diag_rows(Geom g, uint64_t n, const double* __restrict__ k, const double* __restrict__ kref,
                            double sc, double* diag) {
  const uint64_t row = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x;
  if (row >= n) return;
  double d = 0.0;
  row_entries(row, g, k, kref, sc, [&](uint32_t, uint32_t c, double v) {
    if (c == row) d = v;
  });
  diag[row] = d;
}

static Geom geom_of(const fb_mg* m, int lvl) {
  Geom g;
  g.dim = m->dim; g.p = m->degree;
  g.N = 1u << lvl;
  g.M = uint32_t(m->degree) << lvl;
  g.M1 = g.M + 1;
  return g;
}

// CSR prolongation and restriction between level i and the next coarser one (tensor products
// of the 1D interpolation, grid_transfer.hpp:304-321 on nested spaces)
static int build_transfer(fb_mg* m, int i) {
  const int lvl = m->L[i].lvl_num;
  const Geom gf = geom_of(m, lvl), gc = geom_of(m, lvl - 1);
  std::vector<uint32_t> rp, ci, trp, tci;
  std::vector<double> va, tva;
  prol1d(m->degree, gf.M, rp, ci, va);
  transpose1d(gf.M1, gc.M1, rp, ci, va, trp, tci, tva);
  FB_TRY(build_kron(m, m->L[i].P, m->dim, gf.M1, gc.M1, rp, ci, va));
  return build_kron(m, m->L[i].R, m->dim, gc.M1, gf.M1, trp, tci, tva);
}

int ensure_assembled(fb_mg* m, bool matrices, bool transfers) {
  if (!m->structured) return FB_OK;
  for (int i = 0; i < (int)m->L.size(); ++i) {
    Level& L = m->L[i];
    if (matrices && L.lazy_matrix) {
      FB_TRY(build_level_values(m, L, geom_of(m, L.lvl_num), elem_scale(m->dim, L.lvl_num)));
      L.lazy_matrix = false;
    }
    if (transfers && L.lazy_transfer) {
      FB_TRY(build_transfer(m, i));
      L.lazy_transfer = false;
    }
  }
  FB_CUDA(cudaStreamSynchronize(m->stream));
  return FB_OK;
}

}  // namespace fb

using namespace fb;

extern "C" {

int fb_mg_create_structured(fb_mg** out, const fb_structured_desc* d) {
  if (!out || !d) return FB_ERR_INVALID;
  *out = nullptr;
  if ((d->dim != 2 && d->dim != 3) || (d->degree != 1 && d->degree != 2) || d->level_min < 0 ||
      d->level < d->level_min || d->level - d->level_min + 1 > kMaxLevels || d->level > 14)
    return FB_ERR_INVALID;
  {
    const uint64_t M1 = (uint64_t(d->degree) << d->level) + 1;
    const uint64_t n = M1 * M1 * (d->dim == 3 ? M1 : 1);
    const uint64_t row_max = d->dim == 3 ? (d->degree == 1 ? 27 : 125) : (d->degree == 1 ? 9 : 25);
    if (n * row_max >= 0xffffffffull) return FB_ERR_INVALID;  // 32-bit slot addressing
    if (d->degree == 2 && (d->level_min < 1)) return FB_ERR_INVALID;  // Q2 transfer needs >= 2 cells
    if (d->numbering != FB_NUMBERING_LATTICE && d->numbering != FB_NUMBERING_FEAT) return FB_ERR_INVALID;
  }
  fb_mg* m = new fb_mg();
  int st = common_init(m);
  if (st != FB_OK) { fb_mg_destroy(m); return st; }
  m->structured = true;
  m->dim = d->dim; m->degree = d->degree; m->level = d->level; m->level_min = d->level_min;
  build_kref(m->dim, m->degree, m->kref_h, m->nloc);
  if (m->degree == 1) {
    // the cube's reflections give K_ref[a][b] = K_ref[0][a ^ b]; check it before relying on it
    double mx = 0.0, dev = 0.0;
    for (int a = 0; a < m->nloc; ++a)
      for (int b = 0; b < m->nloc; ++b) {
        mx = std::max(mx, std::fabs(m->kref_h[a * m->nloc + b]));
        dev = std::max(dev, std::fabs(m->kref_h[a * m->nloc + b] - m->kref_h[a ^ b]));
      }
    m->mf_ok = dev <= 1e-14 * mx;
    if (m->dim == 3)
      m->mf_faces0 = std::fabs(m->kref_h[1]) <= 1e-14 * mx && std::fabs(m->kref_h[2]) <= 1e-14 * mx &&
                     std::fabs(m->kref_h[4]) <= 1e-14 * mx;
  }
  const int nl = d->level - d->level_min + 1;
  m->L.resize(nl);
  do {
    st = dupload(m, &m->kref, m->kref_h.data(), m->kref_h.size());
    if (st != FB_OK) break;
    if (d->numbering == FB_NUMBERING_FEAT) {
      // the finest level's DOF and cell numbering of FEAT's refined unit square / cube
      const Geom g = geom_of(m, d->level);
      const uint64_t n = uint64_t(g.M1) * g.M1 * (m->dim == 3 ? g.M1 : 1);
      const uint64_t ne = uint64_t(g.N) * g.N * (m->dim == 3 ? g.N : 1);
      if ((st = dalloc(m, &m->feat_dof, n)) != FB_OK || (st = dalloc(m, &m->feat_cell, ne)) != FB_OK) break;
      st = feat_numbering(m->dim, m->degree, d->level, m->feat_dof, m->feat_cell, m->stream);
      if (st != FB_OK) break;
    }
    // coefficients, finest first
    for (int i = 0; i < nl && st == FB_OK; ++i) {
      const int lvl = d->level - i;
      Level& L = m->L[i];
      const Geom g = geom_of(m, lvl);
      L.N = int(g.N);
      L.ne = uint64_t(g.N) * g.N * (m->dim == 3 ? g.N : 1);
      L.n = uint32_t(uint64_t(g.M1) * g.M1 * (m->dim == 3 ? g.M1 : 1));
      if (d->k) {
        st = dalloc(m, &L.k, L.ne);
        if (st != FB_OK) break;
        if (i == 0) {
          // stream-ordered copy; a device-side k must be complete before this call (the caller's stream)
          double* dst = L.k;
          if (m->feat_cell && (st = dalloc(m, &m->pcell, L.ne)) != FB_OK) break;
          if (m->feat_cell) dst = m->pcell;  // FEAT cell order: staged, then permuted
          if (cudaMemcpyAsync(dst, d->k, sizeof(double) * L.ne, d->k_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                              m->stream) != cudaSuccess ||
              cudaStreamSynchronize(m->stream) != cudaSuccess) { st = FB_ERR_CUDA; break; }
          if (m->feat_cell) st = perm_to_lattice(m, L.k, m->pcell, m->feat_cell, L.ne);
        } else {
          k_coarsen_k<<<grid_for(L.ne, 256), 256, 0, m->stream>>>(m->dim, g.N, m->L[i - 1].k, L.k);
          if (cudaGetLastError() != cudaSuccess) st = FB_ERR_CUDA;
        }
      }
    }
    if (st != FB_OK) break;
    for (int i = 0; i < nl && st == FB_OK; ++i) {
      const int lvl = d->level - i;
      Level& L = m->L[i];
      L.lvl_num = lvl;
      // large 3D Q1 levels: structure now, assembled values on first use (ensure_assembled)
      L.lazy_matrix = m->dim == 3 && m->degree == 1 && m->mf_ok && L.n >= kLazyRows;
      st = L.lazy_matrix ? build_level_meta(m, L, geom_of(m, lvl)) : build_level(m, L, geom_of(m, lvl), elem_scale(m->dim, lvl));
      // the level's diagonal from the row gather (the SELL's diagonal entries, bit for bit)
      if (st == FB_OK) st = dalloc(m, &L.diag, L.n);
      if (st == FB_OK) {
        k_diag_rows<<<grid_for(L.n, 128), 128, 0, m->stream>>>(geom_of(m, lvl), L.n, L.k, m->kref,
                                                              elem_scale(m->dim, lvl), L.diag);
        if (cudaGetLastError() != cudaSuccess) st = FB_ERR_CUDA;
      }
    }
    if (st != FB_OK) break;
    // matrix-free operator data of the Q1 levels
    for (int i = 0; i < nl && st == FB_OK && m->mf_ok && m->L[i].St.S; ++i) {
      Level& L = m->L[i];
      const double sc = elem_scale(m->dim, d->level - i);
      L.mf = true;
      L.M1 = geom_of(m, d->level - i).M1;
      for (int r = 0; r < m->nloc; ++r) {
        L.kr64[r] = sc * m->kref_h[r];
        L.kr32[r] = float(L.kr64[r]);
      }
      if (L.k) {
        st = dalloc(m, &L.k32, L.ne);
        if (st != FB_OK) break;
        k_to_f32<<<grid_for(L.ne, 256), 256, 0, m->stream>>>(L.k32, L.k, L.ne);
        if (cudaGetLastError() != cudaSuccess) st = FB_ERR_CUDA;
      }
    }
    if (st != FB_OK) break;
    // transfers (the CSR forms of the large Q1 levels, which only the SELL format uses, on first use)
    for (int i = 0; i + 1 < nl && st == FB_OK; ++i) {
      const int lvl = d->level - i;
      const Geom gf = geom_of(m, lvl), gc = geom_of(m, lvl - 1);
      if (m->degree == 1) {
        Level& Lf = m->L[i];
        Lf.q1_transfer = true;
        Lf.tr.dim = m->dim; Lf.tr.Mf1 = gf.M1; Lf.tr.Mc1 = gc.M1;
        Lf.tr.nf = Lf.n; Lf.tr.nc = m->L[i + 1].n;
      }
      if (m->L[i].lazy_matrix) {
        m->L[i].lazy_transfer = true;
        continue;
      }
      st = build_transfer(m, i);
    }
    if (st != FB_OK) break;
    // coarse direct solver: coarsest level assembled once more on the host
    {
      Level& C = m->L[nl - 1];
      const Geom g = geom_of(m, d->level_min);
      std::vector<double> kc;
      if (C.k) {
        kc.resize(C.ne);
        if (cudaMemcpyAsync(kc.data(), C.k, sizeof(double) * C.ne, cudaMemcpyDeviceToHost, m->stream) != cudaSuccess ||
            cudaStreamSynchronize(m->stream) != cudaSuccess) { st = FB_ERR_CUDA; break; }
      }
      HostCsr h;
      h.rows = h.cols = C.n;
      h.rp.assign(C.n + 1, 0);
      const double sc = elem_scale(m->dim, d->level_min);
      std::vector<uint32_t> filt;
      for (uint64_t r = 0; r < C.n; ++r) {
        row_entries(r, g, kc.empty() ? nullptr : kc.data(), m->kref_h.data(), sc, [&](uint32_t, uint32_t c, double v) {
          h.ci.push_back(c); h.va.push_back(v);
        });
        h.rp[r + 1] = h.ci.size();
        uint32_t cc[3];
        lat_coords(r, g, cc);
        bool bd = false;
        for (int dd = 0; dd < g.dim; ++dd) bd = bd || cc[dd] == 0 || cc[dd] == g.M;
        if (bd) filt.push_back(uint32_t(r));
      }
      if (C.n <= 4096) st = build_coarse_inverse(m, h, filt);
      if (st == FB_OK) st = upload_coarse_csr(m, h);
    }
    if (st != FB_OK) break;
    st = finish_levels(m);
  } while (false);
  if (st != FB_OK) { fb_mg_destroy(m); return st; }
  *out = m;
  return FB_OK;
}

int fb_mg_assemble_rhs(fb_mg* m, int kind, double* rhs) {
  if (!m || !rhs || kind < 0 || kind > 2) return FB_ERR_INVALID;
  if (!m->structured) return FB_ERR_UNSUPPORTED;
  FB_CUDA(cudaSetDevice(m->device));
  const Geom g = geom_of(m, m->level);
  const uint32_t n = m->L[0].n;
  double* out = rhs;
  if (m->feat_dof) {
    if (!m->pv1) FB_TRY(dalloc(m, &m->pv1, n));
    out = m->pv1;
  }
  k_rhs<<<grid_for(n, 128), 128, 0, m->stream>>>(g, n, kind, m->L[0].mask, out);
  FB_CHECK_LAUNCH();
  if (m->feat_dof) FB_TRY(perm_from_lattice(m, rhs, out, m->feat_dof, n));
  FB_CUDA(cudaStreamSynchronize(m->stream));
  return FB_OK;
}

int fb_mg_export_csr(fb_mg* m, int l, uint64_t* rp, uint32_t* col, double* val) {
  if (!m || l < 0 || l >= (int)m->L.size() || !rp || !col || !val) return FB_ERR_INVALID;
  FB_CUDA(cudaSetDevice(m->device));
  FB_TRY(ensure_assembled(m, true, false));
  FB_CUDA(cudaStreamSynchronize(m->stream));
  const DevSell& S = m->L[l].A;
  std::vector<uint32_t> cs(S.nchunks + 1), rl(S.rows), cc(S.nent), perm;
  std::vector<double> vv(S.nent);
  FB_CUDA(cudaMemcpy(cs.data(), S.cs, sizeof(uint32_t) * cs.size(), cudaMemcpyDeviceToHost));
  FB_CUDA(cudaMemcpy(rl.data(), S.rl, sizeof(uint32_t) * rl.size(), cudaMemcpyDeviceToHost));
  FB_CUDA(cudaMemcpy(cc.data(), S.col, sizeof(uint32_t) * cc.size(), cudaMemcpyDeviceToHost));
  FB_CUDA(cudaMemcpy(vv.data(), S.v64, sizeof(double) * vv.size(), cudaMemcpyDeviceToHost));
  if (S.perm) {
    perm.resize(S.rows);
    FB_CUDA(cudaMemcpy(perm.data(), S.perm, sizeof(uint32_t) * perm.size(), cudaMemcpyDeviceToHost));
  }
  std::vector<uint32_t> slot_of(S.rows);
  for (uint32_t sr = 0; sr < S.rows; ++sr) slot_of[perm.empty() ? sr : perm[sr]] = sr;
  // finest level in FEAT numbering: row f is lattice row feat[f], columns renumbered and sorted
  std::vector<uint32_t> feat, lat_to_feat;
  if (m->feat_dof && l == 0) {
    feat.resize(S.rows);
    lat_to_feat.resize(S.rows);
    FB_CUDA(cudaMemcpy(feat.data(), m->feat_dof, sizeof(uint32_t) * S.rows, cudaMemcpyDeviceToHost));
    for (uint32_t f = 0; f < S.rows; ++f) lat_to_feat[feat[f]] = f;
  }
  rp[0] = 0;
  for (uint32_t r = 0; r < S.rows; ++r) rp[r + 1] = rp[r] + rl[feat.empty() ? r : feat[r]];
  std::vector<std::pair<uint32_t, double>> row;
  for (uint32_t r = 0; r < S.rows; ++r) {
    const uint32_t lr = feat.empty() ? r : feat[r];
    const uint32_t sr = slot_of[lr], c = sr / 32, t = sr % 32;
    row.clear();
    for (uint32_t j = 0; j < rl[lr]; ++j) {
      const uint32_t cl = cc[cs[c] + uint64_t(j) * 32 + t];
      row.emplace_back(feat.empty() ? cl : lat_to_feat[cl], vv[cs[c] + uint64_t(j) * 32 + t]);
    }
    if (!feat.empty()) std::sort(row.begin(), row.end(), [](const std::pair<uint32_t, double>& a, const std::pair<uint32_t, double>& b) { return a.first < b.first; });
    for (uint32_t j = 0; j < rl[lr]; ++j) {
      col[rp[r] + j] = row[j].first;
      val[rp[r] + j] = row[j].second;
    }
  }
  return FB_OK;
}

}  // extern "C"

namespace fb {
// element gradient with u and lam in lattice order; grad in the C-ABI's cell order
static int element_grad_lattice(fb_mg* m, const double* u, const double* lam, double* grad) {
  const Geom g = geom_of(m, m->level);
  const uint64_t ne = m->L[0].ne;
  double* out = grad;
  if (m->feat_cell) {
    if (!m->pcell) FB_TRY(dalloc(m, &m->pcell, ne));
    out = m->pcell;
  }
  k_elem_grad<<<grid_for(ne, 128), 128, 0, m->stream>>>(g, ne, u, lam, m->kref, elem_scale(m->dim, m->level), out);
  FB_CHECK_LAUNCH();
  if (m->feat_cell) FB_TRY(perm_from_lattice(m, grad, out, m->feat_cell, ne));
  FB_CUDA(cudaStreamSynchronize(m->stream));
  return FB_OK;
}

static int ensure_stage(fb_mg* m) {
  const uint32_t n = m->L[0].n;
  if (!m->pv1) FB_TRY(dalloc(m, &m->pv1, n));
  if (!m->pv2) FB_TRY(dalloc(m, &m->pv2, n));
  if (!m->pv3) FB_TRY(dalloc(m, &m->pv3, n));
  return FB_OK;
}
}  // namespace fb

extern "C" {

int fb_mg_element_grad(fb_mg* m, const double* u, const double* lam, double* grad) {
  if (!m || !u || !lam || !grad) return FB_ERR_INVALID;
  if (!m->structured) return FB_ERR_UNSUPPORTED;
  FB_CUDA(cudaSetDevice(m->device));
  FB_TRY(ensure_stage(m));
  const double *ul, *laml;
  FB_TRY(in_lattice(m, u, m->pv1, &ul));
  FB_TRY(in_lattice(m, lam, m->pv2, &laml));
  return element_grad_lattice(m, ul, laml, grad);
}

int fb_mg_adjoint_grad(fb_mg* m, const double* u, const double* ut, double* lam, double* grad, fb_solve_info* info) {
  if (!m || !u || !ut || !lam || !grad) return FB_ERR_INVALID;
  if (!m->structured) return FB_ERR_UNSUPPORTED;
  if (!m->configured) return FB_ERR_NOT_READY;
  FB_CUDA(cudaSetDevice(m->device));
  const uint32_t n = m->L[0].n;
  if (!m->adj) FB_TRY(dalloc(m, &m->adj, n));
  FB_TRY(ensure_stage(m));
  // everything below in lattice order; lam and grad leave in the C-ABI's numbering
  const double *ul, *utl;
  FB_TRY(in_lattice(m, u, m->pv1, &ul));
  FB_TRY(in_lattice(m, ut, m->pv2, &utl));
  double* laml = m->feat_dof ? m->pv3 : lam;
  k_adj_rhs<<<ew_grid(n), 256, 0, m->stream>>>(m->adj, ul, utl, m->L[0].mask, n);
  FB_CHECK_LAUNCH();
  FB_CUDA(cudaMemsetAsync(laml, 0, sizeof(double) * n, m->stream));
  // A is symmetric and R = P^T, so the transposed MG-PCG is the configured solver itself
  FB_TRY(solve_dev(m, m->adj, laml, nullptr, info, false));
  if (m->feat_dof) FB_TRY(perm_from_lattice(m, lam, laml, m->feat_dof, n));
  return element_grad_lattice(m, ul, laml, grad);
}

}  // extern "C"
