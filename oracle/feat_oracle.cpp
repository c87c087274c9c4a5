// CPU oracle (TEST INFRASTRUCTURE ONLY) -- see feat_oracle.h for scope and citations.
// Plain C++: every loop follows the reference's summation order where the reference
// defines one (CSR row sums, sequential dot products). Loops whose iterations are
// independent (rows of a matrix product, entries of a vector update, rows of the
// assembled matrices, elements) run on OpenMP threads; each iteration computes exactly
// what the serial loop computes, so results do not depend on the thread count. The
// reductions (dot, norm2) stay sequential, in the reference's order.
#include "feat_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <memory>
#include <type_traits>
#include <unordered_map>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

template<typename T> T eps() { return std::numeric_limits<T>::epsilon(); }

// loops shorter than this stay on the calling thread (the coarse levels)
constexpr int64_t kParMin = 1 << 15;

// ------------------------------------------------------------------------------------
// 1D reference-element data, Gauss-Legendre 3 points on [-1,1] (auto-degree:5 ->
// gauss-legendre:3 for hypercubes, kernel/cubature/auto_alias.hpp:63-75)
struct GL3 {
  double x[3], w[3];
  GL3() {
    const double a = std::sqrt(3.0 / 5.0);
    x[0] = -a; x[1] = 0.0; x[2] = a;
    w[0] = 5.0 / 9.0; w[1] = 8.0 / 9.0; w[2] = 5.0 / 9.0;
  }
};

// 1D Lagrange basis on [-1,1]: degree 1 nodes {-1,1}, degree 2 nodes {-1,0,1}
static void basis1d(int p, double t, double* v, double* d) {
  if (p == 1) {
    v[0] = 0.5 * (1.0 - t); v[1] = 0.5 * (1.0 + t);
    d[0] = -0.5; d[1] = 0.5;
  } else {
    v[0] = 0.5 * t * (t - 1.0); v[1] = 1.0 - t * t; v[2] = 0.5 * t * (t + 1.0);
    d[0] = t - 0.5; d[1] = -2.0 * t; d[2] = t + 0.5;
  }
}

template<typename T>
struct CSR {
  int64_t rows = 0, cols = 0;
  std::vector<int64_t> rp;
  std::vector<int32_t> ci;
  std::vector<T> va;
  int64_t nnz() const { return (int64_t)ci.size(); }
};

// r = b*y + a*A*x (apply_generic.hpp:25-70; |b| < eps zeroes r first, r == y allowed)
template<typename T>
void csr_apply(T* r, T a, const T* x, T b, const T* y, const CSR<T>& A) {
  const int64_t n = A.rows;
  const bool zero = std::fabs(b) < eps<T>();
  const int64_t* rp = A.rp.data();
  const int32_t* ci = A.ci.data();
  const T* va = A.va.data();
#pragma omp parallel for schedule(static) if (n >= kParMin)
  for (int64_t row = 0; row < n; ++row) {
    // r is zeroed (|b| < eps) or set to y before the product, row by row as the reference
    // does array-wide; each row reads only its own r entry
    const T rr = zero ? T(0) : y[row];
    T sum(0);
    for (int64_t k = rp[row]; k < rp[row + 1]; ++k) sum += va[k] * x[ci[k]];
    r[row] = (sum * a) + (b * rr);
  }
}

template<typename T>
T dot(const T* x, const T* y, int64_t n) {  // dot_product_generic.hpp:21-40
  T r(0);
  for (int64_t i = 0; i < n; ++i) r += x[i] * y[i];
  return r;
}
template<typename T>
T norm2(const T* x, int64_t n) {  // norm_generic.hpp:24-32
  T r(0);
  for (int64_t i = 0; i < n; ++i) r += x[i] * x[i];
  return std::sqrt(r);
}
// this = alpha*x + y, with the |alpha| < eps shortcut of dense_vector.hpp:883-905
template<typename T>
void axpy(T* r, const T* x, const T* y, T alpha, int64_t n) {
  if (std::fabs(alpha) < eps<T>()) {
    if (r != y) {
#pragma omp parallel for schedule(static) if (n >= kParMin)
      for (int64_t i = 0; i < n; ++i) r[i] = y[i];
    }
    return;
  }
#pragma omp parallel for schedule(static) if (n >= kParMin)
  for (int64_t i = 0; i < n; ++i) r[i] = alpha * x[i] + y[i];
}

template<typename T, typename U>
void convert(T* dst, const U* src, int64_t n) {
#pragma omp parallel for schedule(static) if (n >= kParMin)
  for (int64_t i = 0; i < n; ++i) dst[i] = T(src[i]);
}

template<typename T>
void copy_vec(T* dst, const T* src, int64_t n) { convert(dst, src, n); }

// ------------------------------------------------------------------------------------
// structured level
struct LevelD {
  int N = 0;            // cells per side
  int64_t M = 0;        // lattice points per side minus one (= degree*N)
  int64_t n = 0;        // dofs
  int64_t ne = 0;       // elements
  std::vector<double> k;  // per element coefficient
  CSR<double> A, P, R;    // P: from coarser level onto this one
  std::vector<int32_t> filt;
  std::vector<char> dir;
};

}  // namespace

struct or_hier {
  int dim = 2, degree = 1, level = 1, level_min = 0;
  int nloc = 4;
  std::vector<double> kref1;        // unit-coefficient element matrix on [-1,1]^d scaled to h=2
  std::vector<LevelD> lv;           // index = level number
  double h_scale(int l) const {     // element matrix factor (h/2)^(d-2)
    const double h = 1.0 / double(1 << l);
    return std::pow(0.5 * h, double(dim - 2));
  }
};

namespace {

// unit-coefficient element stiffness on [-1,1]^d: K_ij = sum_q w_q grad phi_i . grad phi_j
void build_kref(or_hier& H) {
  const int p = H.degree, q1 = p + 1, d = H.dim;
  int nloc = 1;
  for (int i = 0; i < d; ++i) nloc *= q1;
  H.nloc = nloc;
  H.kref1.assign(size_t(nloc) * nloc, 0.0);
  GL3 g;
  int nq = 1;
  for (int i = 0; i < d; ++i) nq *= 3;
  for (int q = 0; q < nq; ++q) {
    int qi[3] = {q % 3, (q / 3) % 3, q / 9};
    double w = 1.0, v[3][3], dv[3][3];
    for (int a = 0; a < d; ++a) {
      w *= g.w[qi[a]];
      basis1d(p, g.x[qi[a]], v[a], dv[a]);
    }
    std::vector<double> grad(size_t(nloc) * d);
    for (int i = 0; i < nloc; ++i) {
      int li[3] = {i % q1, (i / q1) % q1, i / (q1 * q1)};
      for (int c = 0; c < d; ++c) {
        double gg = 1.0;
        for (int a = 0; a < d; ++a) gg *= (a == c) ? dv[a][li[a]] : v[a][li[a]];
        grad[size_t(i) * d + c] = gg;
      }
    }
    for (int i = 0; i < nloc; ++i)
      for (int j = 0; j < nloc; ++j) {
        double s = 0.0;
        for (int c = 0; c < d; ++c) s += grad[size_t(j) * d + c] * grad[size_t(i) * d + c];
        H.kref1[size_t(i) * nloc + j] += w * s;
      }
  }
}

// lattice index of local dof `a` of element e on a level
inline int64_t elem_dof(const or_hier& H, const LevelD& L, int64_t e, int a) {
  const int q1 = H.degree + 1;
  const int64_t N = L.N, M1 = L.M + 1;
  int64_t ex = e % N, ey = (e / N) % N, ez = (H.dim == 3) ? e / (N * N) : 0;
  int ax = a % q1, ay = (a / q1) % q1, az = a / (q1 * q1);
  int64_t X = ex * H.degree + ax, Y = ey * H.degree + ay, Z = ez * H.degree + az;
  return X + M1 * (Y + M1 * Z);
}

// elements containing lattice coordinate X along one direction (element ex spans the lattice
// points [p*ex, p*ex + p]) and the lattice range their dofs cover
struct Span1 { int64_t e0, e1, c0, c1; };
inline Span1 span1(int64_t X, int p, int64_t N) {
  Span1 s;
  s.e0 = std::max<int64_t>(0, (X + p - 1) / p - 1);
  s.e1 = std::min<int64_t>(N - 1, X / p);
  s.c0 = int64_t(p) * s.e0;
  s.c1 = int64_t(p) * s.e1 + p;
  return s;
}

// Assembly of the structured level (bilinear_operator_assembler.hpp:218-339, pattern of
// symbolic_assembler.hpp assemble_matrix_std1). The reference scatters k_e*K_e element by
// element into the CSR rows; here each row gathers the same products from the elements that
// contain it, in ascending element order, so every entry receives the same terms in the same
// order as the scatter (bit-identical), with the rows independent of each other. The row's
// columns are the union of its elements' dofs: per direction a contiguous lattice range, so the
// row is the tensor product of three ranges and lexicographic order is ascending column order.
void build_level(or_hier& H, LevelD& L) {
  const int d = H.dim, p = H.degree, q1 = p + 1;
  const int64_t M1 = L.M + 1, N = L.N;
  L.n = 1; L.ne = 1;
  for (int a = 0; a < d; ++a) { L.n *= M1; L.ne *= N; }
  const int nloc = H.nloc;
  const int64_t n = L.n;
  auto coords = [&](int64_t i, int64_t* c) {
    c[0] = i % M1; c[1] = (i / M1) % M1; c[2] = (d == 3) ? i / (M1 * M1) : 0;
  };
  CSR<double>& A = L.A;
  A.rows = A.cols = n;
  A.rp.assign(n + 1, 0);
#pragma omp parallel for schedule(static) if (n >= kParMin)
  for (int64_t i = 0; i < n; ++i) {
    int64_t c[3];
    coords(i, c);
    int64_t w = 1;
    for (int a = 0; a < d; ++a) { const Span1 s = span1(c[a], p, N); w *= s.c1 - s.c0 + 1; }
    A.rp[i + 1] = w;
  }
  for (int64_t i = 0; i < n; ++i) A.rp[i + 1] += A.rp[i];
  A.ci.resize(A.rp[n]);
  A.va.assign(A.rp[n], 0.0);
  const int lvl = (int)std::lround(std::log2((double)N));
  const double sc = H.h_scale(lvl);
#pragma omp parallel for schedule(static) if (n >= kParMin)
  for (int64_t i = 0; i < n; ++i) {
    int64_t c[3];
    coords(i, c);
    Span1 s[3] = {span1(c[0], p, N), span1(c[1], p, N), {0, 0, 0, 0}};
    s[2] = (d == 3) ? span1(c[2], p, N) : Span1{0, 0, 0, 0};
    const int64_t wx = s[0].c1 - s[0].c0 + 1, wy = s[1].c1 - s[1].c0 + 1, wz = s[2].c1 - s[2].c0 + 1;
    int32_t* ci = A.ci.data() + A.rp[i];
    double* va = A.va.data() + A.rp[i];
    int64_t pos = 0;
    for (int64_t z = 0; z < wz; ++z)
      for (int64_t y = 0; y < wy; ++y)
        for (int64_t x = 0; x < wx; ++x)
          ci[pos++] = (int32_t)((s[0].c0 + x) + M1 * ((s[1].c0 + y) + M1 * (s[2].c0 + z)));
    for (int64_t ez = s[2].e0; ez <= s[2].e1; ++ez)
      for (int64_t ey = s[1].e0; ey <= s[1].e1; ++ey)
        for (int64_t ex = s[0].e0; ex <= s[0].e1; ++ex) {
          const int64_t e = ex + N * (ey + N * ez);
          const double ke = L.k.empty() ? 1.0 : L.k[e];
          const int ax = int(c[0] - p * ex), ay = int(c[1] - p * ey), az = int(c[2] - p * ez);
          const int a = ax + q1 * (ay + q1 * az);
          for (int b = 0; b < nloc; ++b) {
            const int bx = b % q1, by = (b / q1) % q1, bz = b / (q1 * q1);
            const int64_t px = p * ex + bx - s[0].c0, py = p * ey + by - s[1].c0, pz = p * ez + bz - s[2].c0;
            va[px + wx * (py + wy * pz)] += ke * sc * H.kref1[size_t(a) * nloc + b];
          }
        }
  }
  // filter: all lattice points on the boundary
  L.dir.assign(n, 0);
#pragma omp parallel for schedule(static) if (n >= kParMin)
  for (int64_t i = 0; i < n; ++i) {
    int64_t c[3];
    coords(i, c);
    bool b = false;
    for (int a = 0; a < d; ++a) b = b || c[a] == 0 || c[a] == L.M;
    L.dir[i] = b ? 1 : 0;
  }
  for (int64_t i = 0; i < n; ++i)
    if (L.dir[i]) L.filt.push_back((int32_t)i);
}

// nested-space interpolation weights of a coarse 1D basis at fine lattice offsets.
// Q1: fine point 2j -> coarse j (1); 2j+1 -> j, j+1 (1/2 each).
// Q2: coarse element [2c, 2c+2] in the coarse lattice spans fine lattice [4c, 4c+4];
//     fine offsets 0..4 map to coarse local nodes with the Q2 basis values at t = -1,-1/2,0,1/2,1.
void prol_1d(int degree, int64_t Mf, std::vector<std::vector<std::pair<int32_t, double>>>& w) {
  w.assign(Mf + 1, {});
  if (degree == 1) {
    for (int64_t f = 0; f <= Mf; ++f) {
      if (f % 2 == 0) w[f].push_back({(int32_t)(f / 2), 1.0});
      else { w[f].push_back({(int32_t)(f / 2), 0.5}); w[f].push_back({(int32_t)(f / 2 + 1), 0.5}); }
    }
  } else {
    for (int64_t f = 0; f <= Mf; ++f) {
      const int64_t c = std::min<int64_t>(f / 4, Mf / 4 - 1);  // coarse element index
      const int off = (int)(f - 4 * c);                       // 0..4
      const double t = -1.0 + 0.5 * off;
      double v[3], dv[3];
      basis1d(2, t, v, dv);
      for (int a = 0; a < 3; ++a)
        if (v[a] != 0.0) w[f].push_back({(int32_t)(2 * c + a), v[a]});
    }
  }
}

// P row of fine point i: the tensor product of the 1D weight lists (each ascending in the coarse
// index, so the product taken z, y, x is ascending in the lexicographic column); R = P^T.
void build_prol(or_hier& H, LevelD& Lf, const LevelD& Lc) {
  const int d = H.dim;
  std::vector<std::vector<std::pair<int32_t, double>>> w;
  prol_1d(H.degree, Lf.M, w);
  const int64_t Mf1 = Lf.M + 1, Mc1 = Lc.M + 1, n = Lf.n;
  static const std::vector<std::pair<int32_t, double>> one = {{0, 1.0}};
  auto lists = [&](int64_t i, const std::vector<std::pair<int32_t, double>>** l) {
    l[0] = &w[i % Mf1];
    l[1] = &w[(i / Mf1) % Mf1];
    l[2] = (d == 3) ? &w[i / (Mf1 * Mf1)] : &one;
  };
  CSR<double>& P = Lf.P;
  P.rows = n; P.cols = Lc.n;
  P.rp.assign(n + 1, 0);
#pragma omp parallel for schedule(static) if (n >= kParMin)
  for (int64_t i = 0; i < n; ++i) {
    const std::vector<std::pair<int32_t, double>>* l[3];
    lists(i, l);
    P.rp[i + 1] = int64_t(l[0]->size() * l[1]->size() * l[2]->size());
  }
  for (int64_t i = 0; i < n; ++i) P.rp[i + 1] += P.rp[i];
  P.ci.resize(P.rp[n]);
  P.va.resize(P.rp[n]);
#pragma omp parallel for schedule(static) if (n >= kParMin)
  for (int64_t i = 0; i < n; ++i) {
    const std::vector<std::pair<int32_t, double>>* l[3];
    lists(i, l);
    int64_t k = P.rp[i];
    for (auto& z : *l[2])
      for (auto& y : *l[1])
        for (auto& x : *l[0]) {
          P.ci[k] = (int32_t)(x.first + Mc1 * (y.first + Mc1 * z.first));
          P.va[k] = x.second * y.second * z.second;
          ++k;
        }
  }
  // R = P^T (sparse_matrix_csr.hpp transpose): entries of a coarse row ascending in the fine row
  CSR<double>& R = Lf.R;
  R.rows = Lc.n; R.cols = n;
  R.rp.assign(Lc.n + 1, 0);
  for (auto c : P.ci) R.rp[c + 1]++;
  for (int64_t i = 0; i < Lc.n; ++i) R.rp[i + 1] += R.rp[i];
  R.ci.resize(P.ci.size()); R.va.resize(P.va.size());
  std::vector<int64_t> pos(R.rp.begin(), R.rp.end() - 1);
  for (int64_t i = 0; i < n; ++i)
    for (int64_t k = P.rp[i]; k < P.rp[i + 1]; ++k) {
      const int64_t dst = pos[P.ci[k]]++;
      R.ci[dst] = (int32_t)i; R.va[dst] = P.va[k];
    }
}

// ------------------------------------------------------------------------------------
// typed multigrid level (FP64 or FP32 inner)
template<typename T>
struct MGLevel {
  // FP64 levels use the hierarchy's matrices; converted (FP32 / FP16-quantised) levels own copies
  CSR<T> A_own, P_own, R_own;
  const CSR<T>* A = nullptr;
  const CSR<T>* P = nullptr;
  const CSR<T>* R = nullptr;
  std::vector<T> inv_diag;
  const std::vector<int32_t>* filt = nullptr;
  std::vector<T> sol, rhs, def, cor, tmp;
  // smoother scratch
  std::vector<T> s_def, s_cor;
  // coarse direct solver (dense LU of filtered matrix)
  std::vector<double> lu;
  std::vector<int64_t> piv;
};

template<typename T>
void filter_zero(T* v, const std::vector<int32_t>& f) {
  const int64_t n = (int64_t)f.size();
  const int32_t* idx = f.data();
#pragma omp parallel for schedule(static) if (n >= kParMin)
  for (int64_t i = 0; i < n; ++i) v[idx[i]] = T(0);
}

template<typename T>
void fill_vec(T* v, T x, int64_t n) {
#pragma omp parallel for schedule(static) if (n >= kParMin)
  for (int64_t i = 0; i < n; ++i) v[i] = x;
}

template<typename T>
void cast_csr(const CSR<double>& a, CSR<T>& r, int quant) {
  r.rows = a.rows; r.cols = a.cols; r.rp = a.rp; r.ci = a.ci;
  const int64_t nz = (int64_t)a.va.size();
  r.va.resize(nz);
  if (quant == 2) {
    double amax = 0.0;  // max is exact, so the reduction order does not matter
#pragma omp parallel for schedule(static) reduction(max : amax) if (nz >= kParMin)
    for (int64_t i = 0; i < nz; ++i) amax = std::max(amax, std::fabs(a.va[i]));
    const double scale = (amax > 0.0) ? amax / 16384.0 : 1.0;
    const double inv = 1.0 / scale;
#pragma omp parallel for schedule(static) if (nz >= kParMin)
    for (int64_t i = 0; i < nz; ++i) {
      _Float16 h = (_Float16)(a.va[i] * inv);
      r.va[i] = T(float(h) * float(scale));
    }
  } else {
    convert(r.va.data(), a.va.data(), nz);
  }
}

// the level's matrix as the multigrid uses it: the hierarchy's own FP64 matrix, or a converted copy
template<typename T>
const CSR<T>* view_or_cast(const CSR<double>& a, CSR<T>& own, int quant) {
  if constexpr (std::is_same<T, double>::value) {
    if (quant == 0) return &a;
  }
  cast_csr<T>(a, own, quant);
  return &own;
}

template<typename T>
struct MG {
  const or_hier* H;
  or_cfg cfg;
  std::vector<MGLevel<T>> L;  // index 0 = finest
  int nl = 0;

  MG(const or_hier* h, const or_cfg& c) : H(h), cfg(c) {
    nl = h->level - h->level_min + 1;
    L.resize(nl);
    const int quant = (std::is_same<T, float>::value && c.inner == 2) ? 2 : 0;
    for (int i = 0; i < nl; ++i) {
      const LevelD& src = h->lv[h->level - i];
      MGLevel<T>& m = L[i];
      m.A = view_or_cast(src.A, m.A_own, quant);
      if (i + 1 < nl) { m.P = view_or_cast(src.P, m.P_own, 0); m.R = view_or_cast(src.R, m.R_own, 0); }
      m.filt = &src.filt;
      const int64_t n = src.n;
      // Jacobi init: extract diag, invert with omega (jacobi_precond.hpp:137-144)
      m.inv_diag.assign(n, T(0));
      const CSR<T>& Am = *m.A;
#pragma omp parallel for schedule(static) if (n >= kParMin)
      for (int64_t r = 0; r < n; ++r) {
        for (int64_t k = Am.rp[r]; k < Am.rp[r + 1]; ++k)
          if (Am.ci[k] == r) m.inv_diag[r] = Am.va[k];
        m.inv_diag[r] = T(c.omega_jac) / m.inv_diag[r];
      }
      m.sol.assign(n, T(0)); m.rhs = m.def = m.cor = m.tmp = m.s_def = m.s_cor = m.sol;
    }
    if (c.coarse == 0) init_direct(L[nl - 1]);
  }

  void init_direct(MGLevel<T>& m) {
    const int64_t n = m.A->rows;
    m.lu.assign(size_t(n) * n, 0.0);
    std::vector<char> dir(n, 0);
    for (auto i : *m.filt) dir[i] = 1;
    for (int64_t i = 0; i < n; ++i) {
      if (dir[i]) { m.lu[size_t(i) * n + i] = 1.0; continue; }
      for (int64_t k = m.A->rp[i]; k < m.A->rp[i + 1]; ++k)
        if (!dir[m.A->ci[k]]) m.lu[size_t(i) * n + m.A->ci[k]] = double(m.A->va[k]);
    }
    m.piv.resize(n);
    for (int64_t k = 0; k < n; ++k) {
      int64_t p = k;
      for (int64_t i = k + 1; i < n; ++i)
        if (std::fabs(m.lu[size_t(i) * n + k]) > std::fabs(m.lu[size_t(p) * n + k])) p = i;
      m.piv[k] = p;
      if (p != k) for (int64_t j = 0; j < n; ++j) std::swap(m.lu[size_t(k) * n + j], m.lu[size_t(p) * n + j]);
      const double dd = m.lu[size_t(k) * n + k];
      for (int64_t i = k + 1; i < n; ++i) {
        const double l = (m.lu[size_t(i) * n + k] /= dd);
        for (int64_t j = k + 1; j < n; ++j) m.lu[size_t(i) * n + j] -= l * m.lu[size_t(k) * n + j];
      }
    }
  }

  void apply_direct(MGLevel<T>& m, T* cor, const T* def) {
    const int64_t n = m.A->rows;
    std::vector<double> b(n);
    for (int64_t i = 0; i < n; ++i) b[i] = double(def[i]);
    for (auto i : *m.filt) b[i] = 0.0;
    for (int64_t k = 0; k < n; ++k) if (m.piv[k] != k) std::swap(b[k], b[m.piv[k]]);
    for (int64_t i = 0; i < n; ++i) for (int64_t j = 0; j < i; ++j) b[i] -= m.lu[size_t(i) * n + j] * b[j];
    for (int64_t i = n; i > 0; --i) {
      const int64_t r = i - 1;
      for (int64_t j = r + 1; j < n; ++j) b[r] -= m.lu[size_t(r) * n + j] * b[j];
      b[r] /= m.lu[size_t(r) * n + r];
    }
    for (int64_t i = 0; i < n; ++i) cor[i] = T(b[i]);
    filter_zero(cor, *m.filt);
  }

  // Richardson(Jacobi) smoother apply(cor, def): richardson.hpp:160-226 with
  // min_iter = max_iter = nu (no defect norms except the initial one, iterative.hpp:744-766)
  int smooth(MGLevel<T>& m, T* cor, const T* def) {
    const int64_t n = m.A->rows;
    T* sd = m.s_def.data();
    T* t = m.s_cor.data();
    copy_vec(sd, def, n);
    fill_vec(cor, T(0), n);
    const T d0 = norm2(sd, n);
    if (!std::isfinite(d0)) return 3;
    if (d0 <= eps<T>() * eps<T>()) return 2;
    for (int it = 0; it < cfg.nu; ++it) {
      const T* id = m.inv_diag.data();
#pragma omp parallel for schedule(static) if (n >= kParMin)
      for (int64_t i = 0; i < n; ++i) t[i] = id[i] * sd[i];  // component_product
      filter_zero(t, *m.filt);
      axpy(cor, t, cor, T(cfg.omega_rich), n);
      csr_apply(sd, T(-1), cor, T(1), def, *m.A);
      filter_zero(sd, *m.filt);
    }
    return 5;
  }

  // unpreconditioned PCG coarse solver with default settings (pcg.hpp, iterative.hpp:216-235)
  void coarse_pcg(MGLevel<T>& m, T* x, const T* b) {
    const int64_t n = m.A->rows;
    std::vector<T> r(b, b + n), p(n), q(n);
    std::fill(x, x + n, T(0));
    const T tol = std::sqrt(eps<T>());
    T d0 = norm2(r.data(), n);
    if (!std::isfinite(d0) || d0 <= eps<T>() * eps<T>()) return;
    std::copy(r.begin(), r.end(), p.begin());
    filter_zero(p.data(), *m.filt);
    T gamma = dot(r.data(), p.data(), n);
    for (int it = 1; it <= 100; ++it) {
      csr_apply(q.data(), T(1), p.data(), T(0), q.data(), *m.A);
      filter_zero(q.data(), *m.filt);
      T alpha = gamma / dot(q.data(), p.data(), n);
      axpy(x, p.data(), x, alpha, n);
      axpy(r.data(), q.data(), r.data(), -alpha, n);
      T dc = norm2(r.data(), n);
      if (!std::isfinite(dc)) return;
      if (dc > T(1) / eps<T>() * d0) return;
      if (dc <= tol * d0) return;
      std::vector<T> z(r);
      filter_zero(z.data(), *m.filt);
      T g2 = gamma;
      gamma = dot(r.data(), z.data(), n);
      T beta = gamma / g2;
      axpy(p.data(), p.data(), z.data(), beta, n);
    }
  }

  // restriction from level cur down to the coarse level (multigrid.hpp:1711-1832): the
  // pre-smoother (from zero) runs on every level below cur, and on cur itself only when
  // cur_smooth; otherwise the defect left by the peak smoother is restricted
  void apply_rest(int cur, bool cur_smooth) {
    for (int i = cur; i + 1 < nl; ++i) {
      MGLevel<T>& f = L[i];
      MGLevel<T>& c = L[i + 1];
      if (cur_smooth || i > cur) {
        smooth(f, f.sol.data(), f.rhs.data());
        csr_apply(f.def.data(), T(-1), f.sol.data(), T(1), f.rhs.data(), *f.A);
      }
      filter_zero(f.def.data(), *f.filt);
      csr_apply(c.rhs.data(), T(1), f.def.data(), T(0), c.rhs.data(), *f.R);
      filter_zero(c.rhs.data(), *c.filt);
    }
  }

  // coarse-grid solve on the coarsest level (multigrid.hpp:1524-1587)
  void apply_coarse() {
    MGLevel<T>& cl = L[nl - 1];
    switch (cfg.coarse) {
      case 0: apply_direct(cl, cl.sol.data(), cl.rhs.data()); break;
      case 1: coarse_pcg(cl, cl.sol.data(), cl.rhs.data()); break;
      case 2: smooth(cl, cl.sol.data(), cl.rhs.data()); break;
      default:
        std::copy(cl.rhs.begin(), cl.rhs.end(), cl.sol.begin());
        filter_zero(cl.sol.data(), *cl.filt);
    }
  }

  // prolongation from the coarse level up to level cur (multigrid.hpp:1843-2000), with the
  // fixed (omega = 1) or adaptive coarse-grid correction and post-smoothing on every level
  // above cur, on cur itself only when cur_smooth
  void apply_prol(int cur, bool cur_smooth) {
    for (int i = nl - 2; i >= cur; --i) {
      MGLevel<T>& f = L[i];
      MGLevel<T>& c = L[i + 1];
      const int64_t n = f.A->rows;
      csr_apply(f.cor.data(), T(1), c.sol.data(), T(0), f.cor.data(), *f.P);
      filter_zero(f.cor.data(), *f.filt);
      T omega = T(1);
      if (cfg.cgc != 0) {
        csr_apply(f.tmp.data(), T(1), f.cor.data(), T(0), f.tmp.data(), *f.A);
        filter_zero(f.tmp.data(), *f.filt);
        if (cfg.cgc == 1) omega = dot(f.def.data(), f.cor.data(), n) / dot(f.tmp.data(), f.cor.data(), n);
        else omega = dot(f.def.data(), f.tmp.data(), n) / dot(f.tmp.data(), f.tmp.data(), n);
      }
      axpy(f.sol.data(), f.cor.data(), f.sol.data(), omega, n);
      if (cur_smooth || i > cur) {
        if (cfg.cgc != 0) {
          axpy(f.def.data(), f.tmp.data(), f.def.data(), -omega, n);
        } else {
          csr_apply(f.def.data(), T(-1), f.sol.data(), T(1), f.rhs.data(), *f.A);
          filter_zero(f.def.data(), *f.filt);
        }
        smooth(f, f.cor.data(), f.def.data());
        axpy(f.sol.data(), f.cor.data(), f.sol.data(), T(1), n);
      }
    }
  }

  // peak smoother on level l (multigrid.hpp:1589-1680): defect, one application of the
  // level's (peak = pre = post) smoother to it, correction, defect again
  void smooth_peak(int l) {
    MGLevel<T>& f = L[l];
    const int64_t n = f.A->rows;
    csr_apply(f.def.data(), T(-1), f.sol.data(), T(1), f.rhs.data(), *f.A);
    filter_zero(f.def.data(), *f.filt);
    smooth(f, f.cor.data(), f.def.data());
    filter_zero(f.cor.data(), *f.filt);
    axpy(f.sol.data(), f.cor.data(), f.sol.data(), T(1), n);
    csr_apply(f.def.data(), T(-1), f.sol.data(), T(1), f.rhs.data(), *f.A);
    filter_zero(f.def.data(), *f.filt);
  }

  // MultiGrid::apply (multigrid.hpp:1268-1519): V, F or W cycle
  void vcycle(T* cor_out, const T* def_in) {
    const int64_t n0 = L[0].A->rows;
    copy_vec(L[0].rhs.data(), def_in, n0);
    const int last = nl - 1;
    if (cfg.cycle == 1) {
      apply_rest(0, true);
      for (int peak = last - 1; peak > 0; --peak) {
        apply_coarse();
        apply_prol(peak, false);
        smooth_peak(peak);
        apply_rest(peak, false);
      }
      apply_coarse();
      apply_prol(0, true);
    } else if (cfg.cycle == 2) {
      apply_rest(0, true);
      apply_coarse();
      std::vector<int> cnt(nl, 0);
      const int num_cgs = 1 << last;
      for (int cgs = 1; cgs < num_cgs; ++cgs) {
        int peak = last;
        while (peak > 0)
          if (cnt[--peak] == 0) break;
        for (int i = last - 1; i > peak; --i) cnt[i] = 0;
        ++cnt[peak];
        apply_prol(peak, false);
        smooth_peak(peak);
        apply_rest(peak, false);
        apply_coarse();
      }
      apply_prol(0, true);
    } else {
      apply_rest(0, true);
      apply_coarse();
      apply_prol(0, true);
    }
    copy_vec(cor_out, L[0].sol.data(), n0);
  }
};

// stopping logic of IterativeSolver (iterative.hpp:216-235, 490-505, 791-832)
struct Stop {
  double tol_rel, tol_abs, tol_abs_low = 0.0, div_rel, div_abs;
  int max_iter;
  double def_init = 0.0;
  Stop(double tr, int mi) : tol_rel(tr), max_iter(mi) {
    const double e = eps<double>();
    tol_abs = 1.0 / (e * e);
    div_rel = 1.0 / e;
    div_abs = 1.0 / (e * e);
  }
  int initial(double d) {
    def_init = d;
    if (!std::isfinite(d)) return 3;
    if (d <= eps<double>() * eps<double>()) return 2;
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

// preconditioner: FP64 MG, or ConvertPrecond to an FP32 MG
struct Precond {
  std::unique_ptr<MG<double>> mg64;
  std::unique_ptr<MG<float>> mg32;
  std::vector<float> d32, c32;
  Precond(const or_hier* h, const or_cfg& c) {
    if (c.inner == 0) mg64.reset(new MG<double>(h, c));
    else mg32.reset(new MG<float>(h, c));
  }
  void apply(double* cor, const double* def, int64_t n) {
    if (mg64) { mg64->vcycle(cor, def); return; }
    d32.resize(n); c32.resize(n);
    convert(d32.data(), def, n);
    mg32->vcycle(c32.data(), d32.data());
    convert(cor, c32.data(), n);
  }
};

}  // namespace

// ======================================================================================
extern "C" {

or_hier* or_hier_create(int dim, int degree, int level, int level_min, const double* kfine) {
  if ((dim != 2 && dim != 3) || (degree != 1 && degree != 2) || level < level_min || level_min < 0 || level > 12)
    return nullptr;
  or_hier* H = new or_hier();
  H->dim = dim; H->degree = degree; H->level = level; H->level_min = level_min;
  build_kref(*H);
  H->lv.resize(level + 1);
  for (int l = level_min; l <= level; ++l) {
    H->lv[l].N = 1 << l;
    H->lv[l].M = int64_t(degree) << l;
  }
  if (kfine) {
    int64_t ne = 1;
    for (int a = 0; a < dim; ++a) ne *= (int64_t(1) << level);
    H->lv[level].k.assign(kfine, kfine + ne);
    for (int l = level - 1; l >= level_min; --l) {
      const int64_t Nc = int64_t(1) << l, Nf = 2 * Nc;
      int64_t nec = 1;
      for (int a = 0; a < dim; ++a) nec *= Nc;
      auto& kc = H->lv[l].k;
      const auto& kf = H->lv[l + 1].k;
      kc.assign(nec, 0.0);
#pragma omp parallel for schedule(static) if (nec >= kParMin)
      for (int64_t e = 0; e < nec; ++e) {
        int64_t cx = e % Nc, cy = (e / Nc) % Nc, cz = (dim == 3) ? e / (Nc * Nc) : 0;
        double s = 0.0;
        for (int c = 0; c < (1 << dim); ++c) {
          int64_t fx = 2 * cx + (c & 1), fy = 2 * cy + ((c >> 1) & 1), fz = (dim == 3) ? 2 * cz + ((c >> 2) & 1) : 0;
          s += kf[fx + Nf * (fy + Nf * fz)];
        }
        kc[e] = s / double(1 << dim);
      }
    }
  }
  for (int l = level_min; l <= level; ++l) build_level(*H, H->lv[l]);
  for (int l = level_min + 1; l <= level; ++l) build_prol(*H, H->lv[l], H->lv[l - 1]);
  return H;
}

void or_hier_destroy(or_hier* h) { delete h; }

int64_t or_level_ndofs(const or_hier* h, int l) { return h->lv[l].n; }
int64_t or_level_nnz(const or_hier* h, int l) { return h->lv[l].A.nnz(); }
void or_level_csr(const or_hier* h, int l, int64_t* rp, int32_t* ci, double* va) {
  const auto& A = h->lv[l].A;
  std::copy(A.rp.begin(), A.rp.end(), rp);
  std::copy(A.ci.begin(), A.ci.end(), ci);
  std::copy(A.va.begin(), A.va.end(), va);
}
int64_t or_level_pnnz(const or_hier* h, int l) { return h->lv[l].P.nnz(); }
void or_level_p(const or_hier* h, int l, int64_t* rp, int32_t* ci, double* va) {
  const auto& P = h->lv[l].P;
  std::copy(P.rp.begin(), P.rp.end(), rp);
  std::copy(P.ci.begin(), P.ci.end(), ci);
  std::copy(P.va.begin(), P.va.end(), va);
}
void or_level_r(const or_hier* h, int l, int64_t* rp, int32_t* ci, double* va) {
  const auto& R = h->lv[l].R;
  std::copy(R.rp.begin(), R.rp.end(), rp);
  std::copy(R.ci.begin(), R.ci.end(), ci);
  std::copy(R.va.begin(), R.va.end(), va);
}
int64_t or_level_nfilter(const or_hier* h, int l) { return (int64_t)h->lv[l].filt.size(); }
void or_level_filter(const or_hier* h, int l, int32_t* idx) {
  std::copy(h->lv[l].filt.begin(), h->lv[l].filt.end(), idx);
}
int or_element_matrix(const or_hier* h, int l, double* kref) {
  const double sc = h->h_scale(l);
  for (size_t i = 0; i < h->kref1.size(); ++i) kref[i] = sc * h->kref1[i];
  return h->nloc;
}

void or_rhs(const or_hier* h, int kind, double* rhs) {
  const LevelD& L = h->lv[h->level];
  const int d = h->dim, p = h->degree, q1 = p + 1, nloc = h->nloc;
  GL3 g;
  const double hh = 1.0 / double(L.N);
  const double det = std::pow(0.5 * hh, double(d));
  const double pi = 3.14159265358979323846;
  int nq = 1;
  for (int a = 0; a < d; ++a) nq *= 3;
  auto ebs = [](double x) {
    return (std::exp(-(2.0 * x - 1.0) * (2.0 * x - 1.0)) - std::exp(-1.0)) / (1.0 - std::exp(-1.0));
  };
  auto ebs_xx = [](double x) {
    return (64.0 * x * (1.0 - x) - 8.0) * std::exp(-(2.0 * x - 1.0) * (2.0 * x - 1.0)) / (std::exp(-1.0) - 1.0);
  };
  // element load vectors (independent per element), then each dof sums its elements' entries
  // in ascending element order: the order of the reference's element-by-element scatter
  std::vector<double> LV(size_t(L.ne) * nloc, 0.0);
#pragma omp parallel for schedule(static) if (L.ne >= kParMin)
  for (int64_t e = 0; e < L.ne; ++e) {
    int64_t ec[3] = {e % L.N, (e / L.N) % L.N, (d == 3) ? e / (int64_t(L.N) * L.N) : 0};
    double* lv = LV.data() + size_t(e) * nloc;
    for (int q = 0; q < nq; ++q) {
      int qi[3] = {q % 3, (q / 3) % 3, q / 9};
      double w = det, xq[3], v[3][3], dv[3][3];
      for (int a = 0; a < d; ++a) {
        w *= g.w[qi[a]];
        xq[a] = (double(ec[a]) + 0.5 * (g.x[qi[a]] + 1.0)) * hh;
        basis1d(p, g.x[qi[a]], v[a], dv[a]);
      }
      double f;
      if (kind == 0) {
        f = double(d) * pi * pi;
        for (int a = 0; a < d; ++a) f *= std::sin(pi * xq[a]);
      } else if (kind == 1) {
        f = 1.0;
      } else {
        f = 0.0;
        for (int a = 0; a < d; ++a) {
          double t = ebs_xx(xq[a]);
          for (int b = 0; b < d; ++b) if (b != a) t *= ebs(xq[b]);
          f -= t;
        }
      }
      for (int i = 0; i < nloc; ++i) {
        int li[3] = {i % q1, (i / q1) % q1, i / (q1 * q1)};
        double phi = 1.0;
        for (int a = 0; a < d; ++a) phi *= v[a][li[a]];
        lv[i] += w * f * phi;
      }
    }
  }
  const int64_t M1 = L.M + 1;
#pragma omp parallel for schedule(static) if (L.n >= kParMin)
  for (int64_t i = 0; i < L.n; ++i) {
    const int64_t c[3] = {i % M1, (i / M1) % M1, (d == 3) ? i / (M1 * M1) : 0};
    const Span1 sx = span1(c[0], p, L.N), sy = span1(c[1], p, L.N);
    const Span1 sz = (d == 3) ? span1(c[2], p, L.N) : Span1{0, 0, 0, 0};
    double acc = 0.0;
    for (int64_t ez = sz.e0; ez <= sz.e1; ++ez)
      for (int64_t ey = sy.e0; ey <= sy.e1; ++ey)
        for (int64_t ex = sx.e0; ex <= sx.e1; ++ex) {
          const int64_t e = ex + int64_t(L.N) * (ey + int64_t(L.N) * ez);
          const int a = int(c[0] - p * ex) + q1 * (int(c[1] - p * ey) + q1 * int(c[2] - p * ez));
          acc += LV[size_t(e) * nloc + a];
        }
    rhs[i] = acc;
  }
  for (auto i : L.filt) rhs[i] = 0.0;
}

int or_solve(const or_hier* h, const or_cfg* cfg, const double* rhs, double* sol, double* hist, int* iters) {
  const LevelD& L = h->lv[h->level];
  const int64_t n = L.n;
  const CSR<double>& A = L.A;
  Precond M(h, *cfg);
  Stop st(cfg->tol_rel, cfg->max_iter);
  std::vector<double> r(n), p(n), t(n);
  int it = 0;
  auto rec = [&](double d) { if (hist) hist[it] = d; };
  // correct(): r = b - A x; filter_def (pcg.hpp:158-172)
  csr_apply(r.data(), -1.0, sol, 1.0, rhs, A);
  filter_zero(r.data(), L.filt);
  double d0 = norm2(r.data(), n);
  int status = st.initial(d0);
  rec(d0);
  *iters = 0;
  if (status != 1) return status;
  if (cfg->solver == 0) {
    // PCG::_apply_intern (pcg.hpp:188-287)
    M.apply(p.data(), r.data(), n);
    double gamma = dot(r.data(), p.data(), n);
    while (status == 1) {
      csr_apply(t.data(), 1.0, p.data(), 0.0, t.data(), A);
      filter_zero(t.data(), L.filt);
      const double alpha = gamma / dot(t.data(), p.data(), n);
      axpy(sol, p.data(), sol, alpha, n);
      axpy(r.data(), t.data(), r.data(), -alpha, n);
      ++it;
      const double dc = norm2(r.data(), n);
      rec(dc);
      status = st.analyse(it, dc);
      if (status != 1) break;
      M.apply(t.data(), r.data(), n);
      const double g2 = gamma;
      gamma = dot(r.data(), t.data(), n);
      const double beta = gamma / g2;
      axpy(p.data(), p.data(), t.data(), beta, n);
    }
  } else {
    // Richardson::_apply_intern (richardson.hpp:187-226)
    while (status == 1) {
      M.apply(t.data(), r.data(), n);
      axpy(sol, t.data(), sol, cfg->omega_outer, n);
      csr_apply(r.data(), -1.0, sol, 1.0, rhs, A);
      filter_zero(r.data(), L.filt);
      ++it;
      const double dc = norm2(r.data(), n);
      rec(dc);
      status = st.analyse(it, dc);
    }
  }
  *iters = it;
  return status;
}

void or_vcycle(const or_hier* h, const or_cfg* cfg, const double* def, double* cor) {
  Precond M(h, *cfg);
  M.apply(cor, def, h->lv[h->level].n);
}

void or_element_grad(const or_hier* h, const double* u, const double* lam, double* grad) {
  const LevelD& L = h->lv[h->level];
  const int nloc = h->nloc;
  const double sc = h->h_scale(h->level);
#pragma omp parallel for schedule(static) if (L.ne >= kParMin)
  for (int64_t e = 0; e < L.ne; ++e) {
    int64_t loc[27];
    for (int a = 0; a < nloc; ++a) loc[a] = elem_dof(*h, L, e, a);
    double s = 0.0;
    for (int a = 0; a < nloc; ++a) {
      double ka = 0.0;
      for (int b = 0; b < nloc; ++b) ka += h->kref1[size_t(a) * nloc + b] * u[loc[b]];
      s += lam[loc[a]] * ka;
    }
    grad[e] = -sc * s;
  }
}

void or_csr_apply(double* r, double a, const double* x, double b, const double* y,
                  const double* val, const int32_t* col, const int64_t* rowptr,
                  int64_t rows, int64_t cols, int transposed) {
  const double e = eps<double>();
  const int64_t nout = transposed ? cols : rows;
  if (std::fabs(b) < e) {
    for (int64_t i = 0; i < nout; ++i) r[i] = 0.0;
  } else if (r != y) {
    for (int64_t i = 0; i < nout; ++i) r[i] = y[i];
  }
  if (transposed) {
    const double ba = b / a;
    for (int64_t c = 0; c < cols; ++c) r[c] = ba * r[c];
    for (int64_t row = 0; row < rows; ++row)
      for (int64_t k = rowptr[row]; k < rowptr[row + 1]; ++k) r[col[k]] += val[k] * x[row];
    for (int64_t c = 0; c < cols; ++c) r[c] = a * r[c];
  } else {
    for (int64_t row = 0; row < rows; ++row) {
      double sum = 0.0;
      for (int64_t k = rowptr[row]; k < rowptr[row + 1]; ++k) sum += val[k] * x[col[k]];
      r[row] = (sum * a) + (b * r[row]);
    }
  }
}

int or_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

}  // extern "C"

// ------------------------------------------------------------------------------------------
// FEAT3 mesh numbering of the refined unit square / cube.
//
// Restates the standard refinement of conformal hypercube meshes:
//  * new vertices: the old vertices, then one per edge, quad and hexa (in entity order) at its
//    centre (StandardVertexRefiner, intern/standard_vertex_refiner.hpp:65-110, wrapper :195-253);
//  * new entities of each dimension: the children of edges, then of quads, then of hexas, each
//    parent's children consecutive (IndexRefineShapeWrapper, intern/standard_index_refiner.hpp:
//    2762-2840), with the children's vertex lists of StandardIndexRefiner<Hypercube<d>,c,0>
//    (:1346-1402, 1414-1497, 1505-1602, 1723-1811, 1819-2003, 2011-2174);
//  * the unit cube: vertex i at the bits of i, sub-entities by FaceIndexMapping (face_index_
//    mapping.hpp:119-183, common_factories.hpp:71-235);
//  * DOFs of Lagrange1/Lagrange2: vertices, then edges, quads, hexas, one DOF per entity
//    (DofMappingUniform, kernel/space/dof_mapping_common.hpp:255-330).
// A child's vertex that the reference takes from the parent's edges-at-cell / quads-at-cell
// sets (the vertex born from local edge or face k) is found here by its coordinates: the
// centre of the parent's local edge or face k, as FaceIndexMapping numbers them.
namespace {
namespace numbering {
const int kEdge2[4][2] = {{0, 1}, {2, 3}, {0, 2}, {1, 3}};
const int kEdge3[12][2] = {{0, 1}, {2, 3}, {4, 5}, {6, 7}, {0, 2}, {1, 3}, {4, 6}, {5, 7}, {0, 4}, {1, 5}, {2, 6}, {3, 7}};
const int kFace3[6][4] = {{0, 1, 2, 3}, {4, 5, 6, 7}, {0, 1, 4, 5}, {2, 3, 6, 7}, {0, 2, 4, 6}, {1, 3, 5, 7}};
// local points of a parent: 'v' vertex k, 'e' centre of local edge k, 'q' centre of local
// face k (hexa), 'x' the parent's centre
struct Pt { char t; int k; };
const Pt kQuadEdges[4][2] = {{{'e', 0}, {'x', 0}}, {{'x', 0}, {'e', 1}}, {{'e', 2}, {'x', 0}}, {{'x', 0}, {'e', 3}}};
const Pt kQuadQuads[4][4] = {{{'v', 0}, {'e', 0}, {'e', 2}, {'x', 0}}, {{'e', 0}, {'v', 1}, {'x', 0}, {'e', 3}},
                             {{'e', 2}, {'x', 0}, {'v', 2}, {'e', 1}}, {{'x', 0}, {'e', 3}, {'e', 1}, {'v', 3}}};
const Pt kHexaEdges[6][2] = {{{'q', 0}, {'x', 0}}, {{'x', 0}, {'q', 1}}, {{'q', 2}, {'x', 0}},
                             {{'x', 0}, {'q', 3}}, {{'q', 4}, {'x', 0}}, {{'x', 0}, {'q', 5}}};
const Pt kHexaQuads[12][4] = {
    {{'e', 0}, {'q', 0}, {'q', 2}, {'x', 0}}, {{'q', 0}, {'e', 1}, {'x', 0}, {'q', 3}},
    {{'q', 2}, {'x', 0}, {'e', 2}, {'q', 1}}, {{'x', 0}, {'q', 3}, {'q', 1}, {'e', 3}},
    {{'e', 4}, {'q', 0}, {'q', 4}, {'x', 0}}, {{'q', 0}, {'e', 5}, {'x', 0}, {'q', 5}},
    {{'q', 4}, {'x', 0}, {'e', 6}, {'q', 1}}, {{'x', 0}, {'q', 5}, {'q', 1}, {'e', 7}},
    {{'e', 8}, {'q', 2}, {'q', 4}, {'x', 0}}, {{'q', 2}, {'e', 9}, {'x', 0}, {'q', 5}},
    {{'q', 4}, {'x', 0}, {'e', 10}, {'q', 3}}, {{'x', 0}, {'q', 5}, {'q', 3}, {'e', 11}}};
const Pt kHexaHexas[8][8] = {
    {{'v', 0}, {'e', 0}, {'e', 4}, {'q', 0}, {'e', 8}, {'q', 2}, {'q', 4}, {'x', 0}},
    {{'e', 0}, {'v', 1}, {'q', 0}, {'e', 5}, {'q', 2}, {'e', 9}, {'x', 0}, {'q', 5}},
    {{'e', 4}, {'q', 0}, {'v', 2}, {'e', 1}, {'q', 4}, {'x', 0}, {'e', 10}, {'q', 3}},
    {{'q', 0}, {'e', 5}, {'e', 1}, {'v', 3}, {'x', 0}, {'q', 5}, {'q', 3}, {'e', 11}},
    {{'e', 8}, {'q', 2}, {'q', 4}, {'x', 0}, {'v', 4}, {'e', 2}, {'e', 6}, {'q', 1}},
    {{'q', 2}, {'e', 9}, {'x', 0}, {'q', 5}, {'e', 2}, {'v', 5}, {'q', 1}, {'e', 7}},
    {{'q', 4}, {'x', 0}, {'e', 10}, {'q', 3}, {'e', 6}, {'q', 1}, {'v', 6}, {'e', 3}},
    {{'x', 0}, {'q', 5}, {'q', 3}, {'e', 11}, {'q', 1}, {'e', 7}, {'e', 3}, {'v', 7}}};

struct C3 { int64_t c[3]; };

struct Mesh {
  int dim = 2;
  std::vector<C3> vtx;                         // integer coordinates (resolution R)
  std::vector<std::vector<uint32_t>> ent[4];   // ent[d][i] = vertex list of entity i of dim d (d >= 1)
};

C3 centre(const Mesh& m, const std::vector<uint32_t>& vs, const int* loc, int n) {
  C3 r{{0, 0, 0}};
  for (int i = 0; i < n; ++i)
    for (int a = 0; a < 3; ++a) r.c[a] += m.vtx[vs[loc[i]]].c[a];
  for (int a = 0; a < 3; ++a) r.c[a] /= n;
  return r;
}

C3 point(const Mesh& m, const std::vector<uint32_t>& vs, int pdim, Pt p) {
  static const int all[8] = {0, 1, 2, 3, 4, 5, 6, 7};
  switch (p.t) {
    case 'v': return m.vtx[vs[p.k]];
    case 'e': return centre(m, vs, pdim == 2 ? kEdge2[p.k] : kEdge3[p.k], 2);
    case 'q': return centre(m, vs, kFace3[p.k], 4);
    default: return centre(m, vs, all, 1 << pdim);
  }
}

int64_t key(const C3& c, int64_t R) { return c.c[0] + (R + 1) * (c.c[1] + (R + 1) * c.c[2]); }

Mesh unit_cube(int dim, int64_t R) {
  Mesh m;
  m.dim = dim;
  for (int i = 0; i < (1 << dim); ++i) {
    C3 c{{0, 0, 0}};
    for (int a = 0; a < dim; ++a) c.c[a] = ((i >> a) & 1) * R;
    m.vtx.push_back(c);
  }
  if (dim == 2) {
    for (auto& e : kEdge2) m.ent[1].push_back({uint32_t(e[0]), uint32_t(e[1])});
    m.ent[2].push_back({0, 1, 2, 3});
  } else {
    for (auto& e : kEdge3) m.ent[1].push_back({uint32_t(e[0]), uint32_t(e[1])});
    for (auto& f : kFace3) m.ent[2].push_back({uint32_t(f[0]), uint32_t(f[1]), uint32_t(f[2]), uint32_t(f[3])});
    m.ent[3].push_back({0, 1, 2, 3, 4, 5, 6, 7});
  }
  return m;
}

Mesh refine(const Mesh& m, int64_t R) {
  Mesh f;
  f.dim = m.dim;
  f.vtx = m.vtx;
  static const int all[8] = {0, 1, 2, 3, 4, 5, 6, 7};
  for (int d = 1; d <= m.dim; ++d)
    for (auto& vs : m.ent[d]) f.vtx.push_back(centre(m, vs, all, 1 << d));
  std::unordered_map<int64_t, uint32_t> at;
  for (uint32_t i = 0; i < f.vtx.size(); ++i) at[key(f.vtx[i], R)] = i;
  auto child = [&](const std::vector<uint32_t>& parent, int pdim, const Pt* pts, int n) {
    std::vector<uint32_t> c(n);
    for (int i = 0; i < n; ++i) c[i] = at.at(key(point(m, parent, pdim, pts[i]), R));
    return c;
  };
  // edges: of edges, of quads, of hexas
  for (auto& e : m.ent[1]) {
    const uint32_t x = at.at(key(point(m, e, 1, {'x', 0}), R));
    f.ent[1].push_back({e[0], x});
    f.ent[1].push_back({x, e[1]});
  }
  for (auto& q : m.ent[2])
    for (auto& r : kQuadEdges) f.ent[1].push_back(child(q, 2, r, 2));
  if (m.dim == 3)
    for (auto& h : m.ent[3])
      for (auto& r : kHexaEdges) f.ent[1].push_back(child(h, 3, r, 2));
  // quads: of quads, of hexas
  for (auto& q : m.ent[2])
    for (auto& r : kQuadQuads) f.ent[2].push_back(child(q, 2, r, 4));
  if (m.dim == 3) {
    for (auto& h : m.ent[3])
      for (auto& r : kHexaQuads) f.ent[2].push_back(child(h, 3, r, 4));
    for (auto& h : m.ent[3])
      for (auto& r : kHexaHexas) f.ent[3].push_back(child(h, 3, r, 8));
  }
  return f;
}
}  // namespace numbering
}  // namespace

extern "C" int or_feat_numbering(int dim, int degree, int level, uint32_t* dof_lex, uint32_t* cell_lex) {
  using namespace numbering;
  if ((dim != 2 && dim != 3) || (degree != 1 && degree != 2) || level < 0 || level > (dim == 2 ? 12 : 8)) return -1;
  const int64_t R = int64_t(1) << (level + 1);  // coordinates at twice the level's resolution
  Mesh m = unit_cube(dim, R);
  for (int l = 0; l < level; ++l) m = refine(m, R);
  const int64_t N = int64_t(1) << level;
  if (dof_lex) {
    // DOF coordinates: vertices, then (Q2) the centres of edges, quads, hexas
    std::vector<C3> dofs = m.vtx;
    static const int all[8] = {0, 1, 2, 3, 4, 5, 6, 7};
    if (degree == 2)
      for (int d = 1; d <= dim; ++d)
        for (auto& vs : m.ent[d]) dofs.push_back(centre(m, vs, all, 1 << d));
    const int64_t M = degree * N + 1, scale = 2 / degree;  // lattice points per side, coordinate step
    for (size_t f = 0; f < dofs.size(); ++f) {
      int64_t idx = 0, stride = 1;
      for (int a = 0; a < dim; ++a) { idx += dofs[f].c[a] / scale * stride; stride *= M; }
      dof_lex[f] = uint32_t(idx);
    }
  }
  if (cell_lex) {
    const int64_t h = R / N;
    for (size_t c = 0; c < m.ent[dim].size(); ++c) {
      int64_t lo[3] = {R, R, R};
      for (uint32_t v : m.ent[dim][c])
        for (int a = 0; a < dim; ++a) lo[a] = std::min(lo[a], m.vtx[v].c[a]);
      int64_t idx = 0, stride = 1;
      for (int a = 0; a < dim; ++a) { idx += lo[a] / h * stride; stride *= N; }
      cell_lex[c] = uint32_t(idx);
    }
  }
  return 0;
}
