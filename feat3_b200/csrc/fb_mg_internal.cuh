// Internal types of the multigrid driver shared by fb_mg.cu and fb_assembly.cu.
#pragma once
#include <cstddef>
#include "fb_sell.cuh"

#include <vector>

namespace fb {

constexpr int kMaxLevels = 16;

struct DevScalars {
  double rr;            // ||r||^2 of the outer defect
  unsigned kerr;        // set by a staged kernel whose bounded wait expired; it follows rr so that
  unsigned kerr_pad;    // one 16-byte copy per outer iteration brings both to the host
  double rz;            // latest r . z
  double gamma;         // previous r . z (PCG)
  double qp;            // q . p
  double alpha;         // PCG step length whose x update is still pending (applied with the next
                        // direction update, or after the last iteration); 0 = none
  double alpha_hold;    // the step length held over by an even iteration's direction update (its
                        // x update is applied, before alpha's, by the next odd one); 0 = none
  double lvl[2 * kMaxLevels];  // [2l] ||rhs_l||^2, [2l+1] ||post-smoothing defect_l||^2
  double tmp[8];
  unsigned inject;      // test hook of the staged matrix-free kernel (fb_mg_test_expire_wait)
  unsigned inject_pad;
};
// bytes of the scalar block read back per outer iteration: ||r||^2 and the kernel-wait flag
constexpr size_t kHostScalarBytes = offsetof(DevScalars, kerr_pad) + sizeof(unsigned);
static_assert(offsetof(DevScalars, kerr) == sizeof(double), "the wait flag follows ||r||^2");

struct DevSell {
  uint32_t rows = 0, cols = 0, nchunks = 0;
  uint64_t nent = 0;      // stored entries incl. padding
  uint64_t nnz = 0;       // true nonzeros
  uint32_t *cs = nullptr, *cl = nullptr, *col = nullptr, *perm = nullptr;
  uint32_t* rl = nullptr;   // row lengths (setup / export only)
  double* v64 = nullptr;
  float* v32 = nullptr;
  __half* v16 = nullptr;
  float scale16 = 1.0f;
  SellView view(int prec) const {
    SellView v;
    v.nchunks = nchunks; v.rows = rows; v.cs = cs; v.cl = cl; v.col = col; v.perm = perm;
    v.val = prec == FB_PREC_F64 ? (const void*)v64 : (prec == FB_PREC_F32 ? (const void*)v32 : (const void*)v16);
    v.scale = prec == FB_PREC_F16 ? scale16 : 1.0f;
    return v;
  }
};

struct DevCsr {
  uint32_t rows = 0, cols = 0;
  uint64_t nnz = 0;
  uint32_t *rp = nullptr, *col = nullptr;
  double* v64 = nullptr;
  float* v32 = nullptr;
  CsrView view(bool f32) const {
    CsrView v; v.rows = rows; v.rp = rp; v.col = col; v.val = f32 ? (const void*)v32 : (const void*)v64;
    return v;
  }
};

struct DevStencil {
  int S = 0;                 // stencil size (0 = not available on this level)
  int32_t off[27] = {0};     // neighbour offsets in ascending order
  uint32_t nchunks = 0;
  double* v64 = nullptr;
  float* v32 = nullptr;
  __half* v16 = nullptr;
  float scale16 = 1.0f;
};

struct Level {
  uint32_t n = 0;
  DevStencil St;         // implicit-column copy of A (structured Q1 only)
  bool q1_transfer = false;
  Q1Transfer tr;         // matrix-free transfer between this level and the next coarser one
  DevSell A;
  DevCsr P, R;           // P: this level <- next coarser level; R: next coarser <- this
  double* diag = nullptr;
  double* invd64 = nullptr;
  float* invd32 = nullptr;
  uint32_t* mask = nullptr;
  bool mask_boundary = false;  // the mask is exactly the lattice boundary (structured levels)
  uint32_t* filt = nullptr;
  uint32_t nfilt = 0;
  double *rhs64 = nullptr, *x64 = nullptr, *y64 = nullptr, *def64 = nullptr;
  float *rhs32 = nullptr, *x32 = nullptr, *y32 = nullptr, *def32 = nullptr;
  double *cor64 = nullptr, *tmp64 = nullptr;  // adaptive coarse-grid correction: P x_c and A P x_c
  float *cor32 = nullptr, *tmp32 = nullptr;
  // structured info
  int N = 0;             // cells per side
  uint64_t ne = 0;       // elements
  double* k = nullptr;   // per-element coefficient (device)
  // matrix-free Q1 operator (structured Q1 levels)
  bool mf = false;
  uint32_t M1 = 0;       // lattice points per side
  double kr64[8] = {0};  // (h/2)^(dim-2) K_ref[0][r]
  float kr32[8] = {0};
  float* k32 = nullptr;  // FP32 copy of k
  // structured 3D Q1 levels of 2^20 rows and more, whose operator runs matrix-free: the assembled
  // copies (SELL and stencil values) and the CSR transfers are built on first use
  // (ensure_assembled), so a matrix-free solve never holds them
  int lvl_num = 0;             // refinement level (structured)
  bool lazy_matrix = false;    // A / St values not built yet
  bool lazy_transfer = false;  // P / R (this level <- the next coarser one) not built yet
};

// builds the deferred assembled matrices (matrices) and CSR transfers (transfers) of a
// structured hierarchy; a no-op for what exists already
int ensure_assembled(fb_mg* m, bool matrices, bool transfers);

}  // namespace fb

struct fb_mg {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::vector<fb::Level> L;      // 0 = finest
  std::vector<void*> allocs;
  fb_solver_cfg cfg;
  bool configured = false;
  int prec_built = -1;           // precision whose buffers exist
  // structured
  bool structured = false;
  int dim = 0, degree = 0, level = 0, level_min = 0;
  int nloc = 0;
  double* kref = nullptr;        // unit-coefficient element matrix on [-1,1]^d (device)
  bool mf_ok = false;            // K_ref[a][b] == K_ref[0][a^b] (Q1 cube symmetry): matrix-free apply possible
  bool mf_faces0 = false;        // 3D: K_ref[0][1], [0][2], [0][4] (edge-adjacent vertices) are of rounding
                                 // size, as for the Laplacian: the tiled kernel leaves those terms out
  std::vector<double> kref_h;
  // coarse level as CSR (for the single-CTA CG coarse solver) and its work vectors
  fb::DevCsr coarse_csr;
  double *cg64 = nullptr;        // 3 vectors (r, p, q) of the coarse size
  float* cg32 = nullptr;
  // coarse direct solver
  uint32_t nc = 0;
  double* cinv64 = nullptr;
  float* cinv32 = nullptr;
  // outer (finest) vectors
  double *r = nullptr, *p = nullptr, *q = nullptr, *z = nullptr, *xb = nullptr, *bb = nullptr;
  float* p32 = nullptr;          // FP32 search direction of the mixed matrix-free form
  double* pb = nullptr;          // second direction buffer: iteration j writes p_j into buffer j & 1
  float* p32b = nullptr;         // (p / p32 for even j, pb / p32b for odd j)
  float* r32 = nullptr;
  // scalars / reduction workspace
  fb::DevScalars* sc = nullptr;
  double* ws = nullptr;
  unsigned* counter = nullptr;
  double* host_rr = nullptr;     // pinned
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  // graphs
  cudaGraphExec_t g_body[2] = {nullptr, nullptr};  // the iteration body for odd and even iterations
  int g_body_key[2] = {-1, -1};
  int launches = 0;
  int body_launches = 0;
  bool top_s1 = false;                   // finest-level first smoothing step already formed (fused)
  bool top_dot = false;                  // the V-cycle's last finest-level step also forms r . z
  unsigned long long* dbg_err = nullptr;  // FB_DEBUG=1: device word for kernel self-checks
  unsigned* kerr = nullptr;               // &sc->kerr: set by a staged kernel whose bounded wait expired
  unsigned* inject = nullptr;             // &sc->inject (test hook)
  double *hb = nullptr, *hx = nullptr;   // staging for the host-buffer solve
  double* adj = nullptr;                 // adjoint right-hand side
  // FEAT numbering at the C-ABI (structured hierarchies created with FB_NUMBERING_FEAT):
  // feat_dof[f] = lattice index of FEAT DOF f on the finest level, feat_cell[c] = lattice index
  // of FEAT cell c; vectors cross the C-ABI in FEAT order and are permuted on the device
  uint32_t* feat_dof = nullptr;
  uint32_t* feat_cell = nullptr;
  double *pv1 = nullptr, *pv2 = nullptr, *pv3 = nullptr;  // lattice-order staging (n each)
  double* pcell = nullptr;                                 // lattice-order staging (cells)
};

namespace fb {
struct HostCsr {
  uint64_t rows = 0, cols = 0;
  std::vector<uint64_t> rp;
  std::vector<uint32_t> ci;
  std::vector<double> va;
};
template<typename T>
int dalloc(fb_mg* m, T** p, uint64_t n) {
  *p = nullptr;
  if (n == 0) n = 1;
  // 64 bytes of slack: staged kernels widen their copies to 16-byte boundaries
  if (cudaMalloc((void**)p, sizeof(T) * n + 64) != cudaSuccess) { *p = nullptr; cudaGetLastError(); return FB_ERR_ALLOC; }
  m->allocs.push_back(*p);
  return FB_OK;
}
// Upload a host array. The copy is issued on the hierarchy's own stream (a non-blocking
// stream: it is NOT ordered after the legacy default stream), so every kernel launched on that
// stream afterwards sees the data; the host array may be released when this returns.
template<typename T>
int dupload(fb_mg* m, T** p, const T* h, uint64_t n) {
  int st = dalloc(m, p, n);
  if (st != FB_OK) return st;
  if (n && (cudaMemcpyAsync(*p, h, sizeof(T) * n, cudaMemcpyHostToDevice, m->stream) != cudaSuccess ||
            cudaStreamSynchronize(m->stream) != cudaSuccess))
    return FB_ERR_CUDA;
  return FB_OK;
}
int common_init(fb_mg* m);
int finish_levels(fb_mg* m);
int build_coarse_inverse(fb_mg* m, const HostCsr& A, const std::vector<uint32_t>& filt);
int upload_coarse_csr(fb_mg* m, const HostCsr& A);
int upload_sell(fb_mg* m, DevSell& S, const HostCsr& A, int sigma);
int upload_csr(fb_mg* m, DevCsr& D, const HostCsr& A);
int upload_filter(fb_mg* m, Level& L, const std::vector<uint32_t>& f);
// feat_io: rhs and sol are in the C-ABI's numbering (FEAT order when m->feat_dof is set)
int solve_dev(fb_mg* m, const double* rhs, double* sol, double* hist, fb_solve_info* info, bool feat_io = true);
unsigned ew_grid(uint64_t n);
int feat_numbering(int dim, int degree, int level, uint32_t* dof_lex, uint32_t* cell_lex, cudaStream_t s);
// dst[perm[i]] = src[i] (FEAT order -> lattice order) and dst[i] = src[perm[i]] (back)
int perm_to_lattice(fb_mg* m, double* dst, const double* src, const uint32_t* perm, uint64_t n);
int perm_from_lattice(fb_mg* m, double* dst, const double* src, const uint32_t* perm, uint64_t n);
// a finest-level vector of the C-ABI in lattice order: src itself, or src permuted into `stage`
int in_lattice(fb_mg* m, const double* src, double* stage, const double** out);
}  // namespace fb
