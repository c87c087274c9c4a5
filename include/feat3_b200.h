/*
 * feat3_b200 -- C-ABI of the B200 (sm_100a) geometric-multigrid Poisson path.
 *
 * Three layers:
 *  1. Operator layer: one entry point per FEAT3 backend function of the LAFEM arch
 *     boundary for Mem::CUDA (the headers of kernel/lafem/arch). A FEAT3 build binds
 *     LAFEM::Arch::<Op><Mem::CUDA> onto these (one forwarding line each), so the reference's
 *     SparseMatrixCSR/SparseMatrixELL::apply, DenseVector::axpy/dot/norm2, UnitFilter and
 *     Transfer containers -- and the MultiGrid/PCG/Richardson templates above them -- run on
 *     these kernels unchanged.
 *  2. Solver layer: a native multigrid driver (hierarchy, fused V-cycle, PCG/Richardson,
 *     mixed precision, adjoint) for callers that hand over a whole hierarchy.
 *  3. Container file I/O: FEAT3's binary and text formats for matrices and vectors, so a
 *     hierarchy written by a FEAT3 application can be loaded into the solver layer (host code).
 *
 * Conventions: all array pointers of the operator layer are DEVICE pointers; index arrays are
 * 32-bit unsigned, or 64-bit unsigned in the *_u64 entry points (FEAT3's default Index), which
 * read the caller's arrays as they are;
 * sizes are uint64_t; `stream` is a cudaStream_t (NULL = legacy default stream, as the
 * reference uses). Every function returns an int status (FB_OK = 0) and never throws.
 * Functions are asynchronous on `stream` unless their name ends in _sync.
 */
#ifndef FEAT3_B200_H
#define FEAT3_B200_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FB_OK 0
#define FB_ERR_INVALID 1      /* bad argument (null pointer, size out of range, bad config) */
#define FB_ERR_CUDA 2         /* a CUDA runtime call or kernel launch failed */
#define FB_ERR_ALLOC 3        /* device or pinned allocation failed */
#define FB_ERR_UNSUPPORTED 4  /* combination not implemented */
#define FB_ERR_NOT_READY 5    /* object not initialised */
#define FB_ERR_TOO_LARGE 6    /* request exceeds a fixed capacity of the entry point */
#define FB_ERR_TIMEOUT 7      /* a bounded wait inside a kernel expired (the context stays usable) */

#if defined(__GNUC__)
#define FB_API __attribute__((visibility("default")))
#else
#define FB_API
#endif

typedef void* fb_stream_t;

/* ===================================================================================== */
/* 1. Operator layer (drop-in for LAFEM::Arch::*<Mem::CUDA>)                             */
/* ===================================================================================== */

/* r = b*y + a*A*x, A in CSR. |b| < eps => y ignored and r = a*A*x. r may alias y.
 * transposed != 0: r (length cols) = b*y + a*A^T*x.
 * Replaces Arch::Apply<Mem::CUDA>::csr (kernel/lafem/arch/apply.hpp:271-275, apply.cu:241-302). */
FB_API int fb_csr_apply_f64(double* r, double a, const double* x, double b, const double* y,
                     const double* val, const uint32_t* col_ind, const uint32_t* row_ptr,
                     uint64_t rows, uint64_t columns, uint64_t used_elements, int transposed,
                     fb_stream_t stream);
FB_API int fb_csr_apply_f32(float* r, float a, const float* x, float b, const float* y,
                     const float* val, const uint32_t* col_ind, const uint32_t* row_ptr,
                     uint64_t rows, uint64_t columns, uint64_t used_elements, int transposed,
                     fb_stream_t stream);
/* The same with 64-bit index arrays, read as they are (FEAT3's default Index is unsigned long,
 * kernel/base_header.hpp:95-97). Replaces the unsigned-long overload of Arch::Apply<Mem::CUDA>::csr
 * (kernel/lafem/arch/apply.hpp:274, apply.cu:25-39,242-269). */
FB_API int fb_csr_apply_f64_u64(double* r, double a, const double* x, double b, const double* y,
                     const double* val, const uint64_t* col_ind, const uint64_t* row_ptr,
                     uint64_t rows, uint64_t columns, uint64_t used_elements, int transposed,
                     fb_stream_t stream);
FB_API int fb_csr_apply_f32_u64(float* r, float a, const float* x, float b, const float* y,
                     const float* val, const uint64_t* col_ind, const uint64_t* row_ptr,
                     uint64_t rows, uint64_t columns, uint64_t used_elements, int transposed,
                     fb_stream_t stream);

/* r = b*y + a*A*x, A in FEAT's SELL-C layout (val/col_ind chunk-major with stride C, cs =
 * chunk starts, cl = chunk lengths). Replaces Arch::Apply<Mem::CUDA>::ell
 * (kernel/lafem/arch/apply.hpp:296, apply.cu:42-61,432-457). */
FB_API int fb_ell_apply_f64(double* r, double a, const double* x, double b, const double* y,
                     const double* val, const uint32_t* col_ind, const uint32_t* cs,
                     const uint32_t* cl, uint64_t C, uint64_t rows, fb_stream_t stream);
FB_API int fb_ell_apply_f32(float* r, float a, const float* x, float b, const float* y,
                     const float* val, const uint32_t* col_ind, const uint32_t* cs,
                     const uint32_t* cl, uint64_t C, uint64_t rows, fb_stream_t stream);
/* The same with 64-bit index arrays: Arch::Apply<Mem::CUDA>::ell<DT_, unsigned long>
 * (kernel/lafem/arch/apply.hpp:296). */
FB_API int fb_ell_apply_f64_u64(double* r, double a, const double* x, double b, const double* y,
                     const double* val, const uint64_t* col_ind, const uint64_t* cs,
                     const uint64_t* cl, uint64_t C, uint64_t rows, fb_stream_t stream);
FB_API int fb_ell_apply_f32_u64(float* r, float a, const float* x, float b, const float* y,
                     const float* val, const uint64_t* col_ind, const uint64_t* cs,
                     const uint64_t* cl, uint64_t C, uint64_t rows, fb_stream_t stream);

/* r = a*x + y; |a| < eps => r = y. Replaces Arch::Axpy<Mem::CUDA>::dv (axpy.cu:23-55)
 * with the shortcut of DenseVector::axpy (kernel/lafem/dense_vector.hpp:883-905). */
FB_API int fb_axpy_f64(double* r, double a, const double* x, const double* y, uint64_t n, fb_stream_t stream);
FB_API int fb_axpy_f32(float* r, float a, const float* x, const float* y, uint64_t n, fb_stream_t stream);

/* *result (device) = x . y, summed in FP64 in a fixed order (deterministic).
 * Replaces Arch::DotProduct<Mem::CUDA>::value (dot_product.cu:24-64). */
FB_API int fb_dot_f64(const double* x, const double* y, uint64_t n, double* result, fb_stream_t stream);
FB_API int fb_dot_f32(const float* x, const float* y, uint64_t n, double* result, fb_stream_t stream);
/* same, returning the value to the host (synchronises `stream`), as the reference's value() */
FB_API int fb_dot_f64_sync(const double* x, const double* y, uint64_t n, double* host_result, fb_stream_t stream);
FB_API int fb_dot_f32_sync(const float* x, const float* y, uint64_t n, double* host_result, fb_stream_t stream);

/* No counterpart in the reference: a variant of fb_dot_f64 that allocates nothing, for callers
 * that cannot call cudaMalloc (an external allocator owns all device memory, or allocation is
 * forbidden after start-up). Its partial sums live in a fixed device array inside the library
 * (FB_NOALLOC_DOT_MAX_CTAS doubles plus a counter, 32 KiB on every GPU that loads the library,
 * held until exit), so n is limited to FB_NOALLOC_DOT_MAX_N elements; larger n returns
 * FB_ERR_TOO_LARGE. The first call on each device looks up the array's device address, and
 * with CUDA's lazy module loading (the default) that lookup may load the library's module,
 * which allocates device memory for its code and arrays: make one warm-up call per device at
 * start-up, before allocation is forbidden and before any stream capture. All calls share
 * the one array: calls that overlap on the GPU (concurrent streams) race and must be
 * serialised by the caller.
 * *result (device) = x . y, as fb_dot_f64. */
#define FB_NOALLOC_DOT_MAX_CTAS 4096
#define FB_NOALLOC_DOT_ELEMS_PER_CTA 16384ull
#define FB_NOALLOC_DOT_MAX_N (4096ull * 16384ull)
FB_API int fb_dot_f64_noalloc(const double* x, const double* y, uint64_t n, double* result, fb_stream_t stream);

/* *result (device) = ||x||_2. Replaces Arch::Norm2<Mem::CUDA>::value (norm.cu:24-60). */
FB_API int fb_norm2_f64(const double* x, uint64_t n, double* result, fb_stream_t stream);
FB_API int fb_norm2_f32(const float* x, uint64_t n, double* result, fb_stream_t stream);
FB_API int fb_norm2_f64_sync(const double* x, uint64_t n, double* host_result, fb_stream_t stream);
FB_API int fb_norm2_f32_sync(const float* x, uint64_t n, double* host_result, fb_stream_t stream);

/* r = x o y. Replaces Arch::ComponentProduct<Mem::CUDA>::value (component_product.cu:20-27). */
FB_API int fb_component_product_f64(double* r, const double* x, const double* y, uint64_t n, fb_stream_t stream);
FB_API int fb_component_product_f32(float* r, const float* x, const float* y, uint64_t n, fb_stream_t stream);
/* r = s / x. Replaces Arch::ComponentInvert<Mem::CUDA>::value (component_invert.cu:20-28). */
FB_API int fb_component_invert_f64(double* r, const double* x, double s, uint64_t n, fb_stream_t stream);
FB_API int fb_component_invert_f32(float* r, const float* x, float s, uint64_t n, fb_stream_t stream);
/* r = s * x. Replaces Arch::Scale<Mem::CUDA>::value (scale.cu:20-27). */
FB_API int fb_scale_f64(double* r, const double* x, double s, uint64_t n, fb_stream_t stream);
FB_API int fb_scale_f32(float* r, const float* x, float s, uint64_t n, fb_stream_t stream);

/* diag[i] = A(i,i) (0 if absent). Replaces Arch::Diagonal<Mem::CUDA>::csr / ::ell
 * (diagonal.cu:20-86). */
FB_API int fb_diagonal_csr_f64(double* diag, const double* val, const uint32_t* col_ind,
                        const uint32_t* row_ptr, uint64_t rows, fb_stream_t stream);
FB_API int fb_diagonal_csr_f32(float* diag, const float* val, const uint32_t* col_ind,
                        const uint32_t* row_ptr, uint64_t rows, fb_stream_t stream);
FB_API int fb_diagonal_ell_f64(double* diag, const double* val, const uint32_t* col_ind, const uint32_t* cs,
                        const uint32_t* cl, uint64_t C, uint64_t rows, fb_stream_t stream);
FB_API int fb_diagonal_ell_f32(float* diag, const float* val, const uint32_t* col_ind, const uint32_t* cs,
                        const uint32_t* cl, uint64_t C, uint64_t rows, fb_stream_t stream);
/* The same with 64-bit index arrays: Arch::Diagonal<Mem::CUDA>::csr / ::ell<DT_, unsigned long>
 * (kernel/lafem/arch/diagonal.hpp:69-80). */
FB_API int fb_diagonal_csr_f64_u64(double* diag, const double* val, const uint64_t* col_ind,
                        const uint64_t* row_ptr, uint64_t rows, fb_stream_t stream);
FB_API int fb_diagonal_csr_f32_u64(float* diag, const float* val, const uint64_t* col_ind,
                        const uint64_t* row_ptr, uint64_t rows, fb_stream_t stream);
FB_API int fb_diagonal_ell_f64_u64(double* diag, const double* val, const uint64_t* col_ind, const uint64_t* cs,
                        const uint64_t* cl, uint64_t C, uint64_t rows, fb_stream_t stream);
FB_API int fb_diagonal_ell_f32_u64(float* diag, const float* val, const uint64_t* col_ind, const uint64_t* cs,
                        const uint64_t* cl, uint64_t C, uint64_t rows, fb_stream_t stream);

/* v[idx[i]] = sv[i] / v[idx[i]] = 0. Replaces Arch::UnitFilter<Mem::CUDA>::filter_rhs /
 * filter_def (unit_filter.cu:21-36; used for filter_sol/filter_cor as well,
 * kernel/lafem/unit_filter.hpp:399-437). */
FB_API int fb_unit_filter_rhs_f64(double* v, const double* sv_elements, const uint32_t* sv_indices, uint64_t ue, fb_stream_t stream);
FB_API int fb_unit_filter_def_f64(double* v, const uint32_t* sv_indices, uint64_t ue, fb_stream_t stream);
FB_API int fb_unit_filter_rhs_f32(float* v, const float* sv_elements, const uint32_t* sv_indices, uint64_t ue, fb_stream_t stream);
FB_API int fb_unit_filter_def_f32(float* v, const uint32_t* sv_indices, uint64_t ue, fb_stream_t stream);
/* The same with 64-bit index lists: Arch::UnitFilter<Mem::CUDA>::filter_rhs / filter_def
 * <DT_, unsigned long> (kernel/lafem/arch/unit_filter.hpp:74-81). */
FB_API int fb_unit_filter_rhs_f64_u64(double* v, const double* sv_elements, const uint64_t* sv_indices, uint64_t ue, fb_stream_t stream);
FB_API int fb_unit_filter_def_f64_u64(double* v, const uint64_t* sv_indices, uint64_t ue, fb_stream_t stream);
FB_API int fb_unit_filter_rhs_f32_u64(float* v, const float* sv_elements, const uint64_t* sv_indices, uint64_t ue, fb_stream_t stream);
FB_API int fb_unit_filter_def_f32_u64(float* v, const uint64_t* sv_indices, uint64_t ue, fb_stream_t stream);

/* precision conversion and fill. Replace MemoryPool<Mem::CUDA>::convert / set_memory
 * (kernel/util/memory_pool.cu:26-41,176-222). */
FB_API int fb_convert_f64_to_f32(float* dst, const double* src, uint64_t n, fb_stream_t stream);
FB_API int fb_convert_f32_to_f64(double* dst, const float* src, uint64_t n, fb_stream_t stream);
FB_API int fb_set_f64(double* dst, double value, uint64_t n, fb_stream_t stream);
FB_API int fb_set_f32(float* dst, float value, uint64_t n, fb_stream_t stream);

/* ===================================================================================== */
/* 2. Solver layer (native MultiGrid / PCG / Richardson driver)                          */
/* ===================================================================================== */

typedef struct fb_mg fb_mg;

/* Structured hierarchy assembled on the device: unit square/cube, `level_min`..`level`
 * (N = 2^level cells per side), Q1 (degree 1) or Q2 (degree 2) Laplace with a per-element
 * coefficient (lexicographic, N^dim values, host or device pointer; NULL = 1; coarse
 * levels use the mean of the 2^dim children), homogeneous Dirichlet boundary, nested
 * interpolation transfers. Follows the assembly of tutorials/tutorial_05_multigrid.cpp:
 * 226-303 on a lexicographic lattice numbering. */
typedef struct fb_structured_desc {
  int dim;            /* 2 or 3 */
  int degree;         /* 1 (Q1) or 2 (Q2) */
  int level;          /* finest level */
  int level_min;      /* coarsest level */
  const double* k;    /* per-element coefficient on the finest level or NULL */
  int k_on_device;    /* 1 if k is a device pointer */
  int sell_sigma;     /* SELL-C-sigma sorting window for the level matrices; 1 = no sorting */
  int numbering;      /* FB_NUMBERING_LATTICE [0] or FB_NUMBERING_FEAT: the order of the finest
                         level's DOFs and cells in every vector the solver layer takes or returns */
} fb_structured_desc;
#define FB_NUMBERING_LATTICE 0  /* lexicographic lattice, x fastest */
#define FB_NUMBERING_FEAT 1     /* FEAT3's numbering of the refined unit square / cube */
FB_API int fb_mg_create_structured(fb_mg** out, const fb_structured_desc* desc);

/* FEAT3's numbering of the unit square (dim 2) or cube (dim 3) refined `level` times by
 * RefinedUnitCubeFactory / StandardRefinery (kernel/geometry/common_factories.hpp:71-235,
 * conformal_mesh.hpp:439-528; the Q1/Q2 DOFs by DofMappingUniform, kernel/space/
 * dof_mapping_common.hpp:255-330), computed on the device without building the mesh:
 * dof_lex[f] = lexicographic lattice index of FEAT DOF f ((degree*2^level+1)^dim entries),
 * cell_lex[c] = lexicographic index of FEAT cell c (2^(dim*level) entries). Device pointers;
 * either may be NULL. Asynchronous on `stream`. */
FB_API int fb_feat_numbering(int dim, int degree, int level, uint32_t* dof_lex, uint32_t* cell_lex,
                             fb_stream_t stream);

/* Hierarchy from caller-supplied CSR matrices (e.g. assembled by FEAT3 on the host in its
 * own numbering): level 0 = finest. Host pointers; copied to the device. P[l] maps level
 * l+1 onto level l (rows = n[l]), R[l] = its transpose (FEAT stores both, transfer.hpp:
 * 249-285). filter[l] = Dirichlet DOF list of level l. Mirrors
 * MultiGridHierarchy::push_level (kernel/solver/multigrid.hpp:633,677). */
typedef struct fb_csr_host {
  uint64_t rows, cols, nnz;
  const uint64_t* row_ptr;  /* rows+1 */
  const uint64_t* col_ind;  /* nnz */
  const double* val;        /* nnz */
} fb_csr_host;
FB_API int fb_mg_create_csr(fb_mg** out, int num_levels, const fb_csr_host* A, const fb_csr_host* P,
                     const fb_csr_host* R, const uint64_t* const* filter, const uint64_t* filter_size,
                     int sell_sigma);

FB_API void fb_mg_destroy(fb_mg* mg);

/* Solver configuration (defaults in brackets), mirroring the composition of
 * applications/poisson_dirichlet.cpp:152-190:
 *   outer  : FB_OUTER_PCG [PCG] or FB_OUTER_RICHARDSON (pcg.hpp:188-287, richardson.hpp:187-226)
 *   nu     : pre = post Richardson(Jacobi) smoothing steps (richardson.hpp, jacobi_precond.hpp)
 *   coarse : FB_COARSE_DIRECT (dense solve of the filtered coarse system), FB_COARSE_PCG
 *            (unpreconditioned CG, default settings), FB_COARSE_SMOOTHER, FB_COARSE_NONE
 *   precision: FB_PREC_F64 (drop-in FP64), FB_PREC_F32 (mixed: FP64 outer defect/update,
 *            FP32 V-cycle), FB_PREC_F16 (as F32 with FP16 matrix values behind a per-level
 *            FP32 scale) -- ConvertPrecond composition (convert_precond.hpp:41-120). */
#define FB_OUTER_PCG 0
#define FB_OUTER_RICHARDSON 1
#define FB_COARSE_DIRECT 0
#define FB_COARSE_PCG 1
#define FB_COARSE_SMOOTHER 2
#define FB_COARSE_NONE 3
#define FB_PREC_F64 0
#define FB_PREC_F32 1
#define FB_PREC_F16 2
/* level-matrix storage of the V-cycle and the outer solver:
 *   FB_FORMAT_SELL    SELL-C-sigma with 32-bit column indices and CSR transfer matrices
 *                     (what a hierarchy handed over by FEAT3 uses);
 *   FB_FORMAT_STENCIL on structured Q1 hierarchies: SELL-32 with implicit stencil columns
 *                     (no index stream) and matrix-free Q1 interpolation/restriction;
 *                     other hierarchies fall back to FB_FORMAT_SELL level by level;
 *   FB_FORMAT_MATFREE on structured Q1 hierarchies: no level matrix is read; every operator
 *                     application (smoothers, defects, the outer solver's products) is formed
 *                     from the per-cell coefficients and the reference element matrix, with
 *                     matrix-free Q1 transfers; other hierarchies fall back as above. */
#define FB_FORMAT_SELL 0
#define FB_FORMAT_STENCIL 1
#define FB_FORMAT_MATFREE 2
typedef struct fb_solver_cfg {
  int outer;
  int nu;
  double omega_jac;
  double omega_rich;
  double omega_outer;
  int coarse;
  double tol_rel;
  int max_iter;
  int precision;
  int use_graphs;     /* capture the per-iteration launch sequence in a CUDA graph */
  int format;         /* FB_FORMAT_SELL, FB_FORMAT_STENCIL or FB_FORMAT_MATFREE */
  int flags;          /* FB_FLAG_*: switch individual fusions off (testing; 0 = all on; any other
                         bit: FB_ERR_INVALID) */
  int cycle;          /* FB_CYCLE_V, FB_CYCLE_F or FB_CYCLE_W (Solver::MultiGridCycle) */
  int adapt_cgc;      /* FB_CGC_FIXED, FB_CGC_MIN_ENERGY or FB_CGC_MIN_DEFECT (Solver::MultiGridAdaptCGC) */
} fb_solver_cfg;
#define FB_CYCLE_V 0
#define FB_CYCLE_F 1
#define FB_CYCLE_W 2
#define FB_CGC_FIXED 0
#define FB_CGC_MIN_ENERGY 1
#define FB_CGC_MIN_DEFECT 2
/* flags: the coarse end of the V-cycle level by level instead of one cluster launch; PCG's
 * r . z as its own reduction instead of inside the last smoothing step; the matrix-free
 * operator without the shared-memory tiled kernel; the two finest 3D matrix-free levels with
 * the line-tiled kernel instead of the streaming one */
#define FB_FLAG_NO_COARSE_FUSION 1
#define FB_FLAG_NO_DOT_FUSION 2
#define FB_FLAG_NO_TILED 4
#define FB_FLAG_NO_STREAM 8
FB_API void fb_solver_cfg_default(fb_solver_cfg* cfg);
FB_API int fb_mg_configure(fb_mg* mg, const fb_solver_cfg* cfg);

/* Result of a solve. status uses the reference's Solver::Status numbering
 * (kernel/solver/base.hpp:48-64): 0 undefined, 1 progress, 2 success, 3 aborted,
 * 4 diverged, 5 max_iter, 6 stagnated. */
typedef struct fb_solve_info {
  int status;
  int iters;
  double def_init;
  double def_final;
  double solve_ms;       /* device time of the solve (CUDA events) */
  int kernel_launches;   /* kernels launched by this solve */
} fb_solve_info;

/* rhs/sol are DEVICE pointers of the finest level's size; sol holds the initial guess.
 * hist (host, may be NULL) receives max_iter+1 defect norms. Equivalent to
 * Solver::solve(PCG(MG), sol, rhs) (kernel/solver/iterative.hpp:926-935). */
FB_API int fb_mg_solve(fb_mg* mg, const double* rhs, double* sol, double* hist, fb_solve_info* info);
/* same with HOST buffers: uploads rhs and sol, solves, downloads sol (end-to-end path) */
FB_API int fb_mg_solve_host(fb_mg* mg, const double* rhs_host, double* sol_host, double* hist, fb_solve_info* info);
/* The same from a zero initial guess (sol_host is output only, so it is not copied to the device;
 * Solver::solve after vec_sol.format()). */
FB_API int fb_mg_solve_host_zero(fb_mg* mg, const double* rhs_host, double* sol_host, double* hist, fb_solve_info* info);
/* one preconditioner application cor = MG(def) on the finest level (device pointers);
 * FB_ERR_TIMEOUT when a bounded wait inside a kernel expired (cor is then not valid) */
FB_API int fb_mg_vcycle(fb_mg* mg, const double* def, double* cor);

/* Load vector of the structured finest level (device output): kind 0 = d*pi^2*prod sin(pi x),
 * 1 = f = 1, 2 = exp-bubble Laplacian (common_functionals.hpp:137-225); filtered. */
FB_API int fb_mg_assemble_rhs(fb_mg* mg, int kind, double* rhs);
FB_API uint64_t fb_mg_num_dofs(const fb_mg* mg, int level);   /* level 0 = finest */
FB_API int fb_mg_num_levels(const fb_mg* mg);
/* copy the finest-level matrix of a structured hierarchy out as CSR (host arrays sized by
 * fb_mg_nnz); for parity tests */
FB_API uint64_t fb_mg_nnz(const fb_mg* mg, int level);
FB_API int fb_mg_export_csr(fb_mg* mg, int level, uint64_t* row_ptr, uint32_t* col_ind, double* val);

/* Adjoint of J(u) = 1/2 ||u - u_target||^2 subject to A(k) u = f on a structured hierarchy:
 * solves the transposed system A^T lambda = filter(u - u_target) with the configured MG
 * solver (A is symmetric, R = P^T, so the transposed V-cycle is the same operator) and
 * evaluates dJ/dk_e = -lambda_e^T K_e^(1) u_e per finest-level element.
 * Device pointers: u, u_target, lambda (out, n dofs), grad (out, N^dim). */
FB_API int fb_mg_adjoint_grad(fb_mg* mg, const double* u, const double* u_target, double* lambda,
                       double* grad, fb_solve_info* info);
/* element gradient only: grad[e] = -lambda_e^T K_e^(1) u_e */
FB_API int fb_mg_element_grad(fb_mg* mg, const double* u, const double* lambda, double* grad);

/* Measurement helper: runs the level-`level` fused SpMV kernel `reps` times on the
 * hierarchy's stream between CUDA events and returns the mean device time per launch.
 * which: 0 = fused defect + Jacobi update (the smoother step), 1 = defect, 2 = PCG q = A p
 * with q.p, 3 = the same from the FP32-stored direction of the mixed matrix-free form (level 0,
 * precision FB_PREC_F32); precision selects the value storage (FB_PREC_*). */
FB_API int fb_mg_time_spmv(fb_mg* mg, int level, int which, int precision, int reps, double* ms_per_launch);

/* Test hook, no counterpart in the reference: arms a one-shot flag so that the next launch of
 * the bulk-staged matrix-free kernel (3D structured levels, FB_FORMAT_MATFREE) leaves one stage
 * of its first block unfilled. The consumers' bounded wait on that stage expires (after about
 * one second), the kernel records it and returns, and the solve in progress stops at its next
 * read-back and returns FB_ERR_TIMEOUT; the handle and the CUDA context stay usable. Nothing but
 * the tests arms it. */
FB_API int fb_mg_test_expire_wait(fb_mg* mg);

/* ===================================================================================== */
/* 3. Container file I/O in FEAT3's formats (host only, no device needed)                */
/* ===================================================================================== */

/* File modes: the values of LAFEM::FileMode (kernel/lafem/base.hpp:31-46). */
#define FB_FILE_EXP 0      /* fm_exp: one value per line (vectors) */
#define FB_FILE_DV 1       /* fm_dv: serialised DenseVector */
#define FB_FILE_MTX 2      /* fm_mtx: MatrixMarket text */
#define FB_FILE_CSR 4      /* fm_csr: serialised SparseMatrixCSR */
#define FB_FILE_BINARY 12  /* fm_binary: the serialised form of the container type */
#define FB_ERR_IO 8        /* a file could not be opened, read or written */
#define FB_ERR_FORMAT 9    /* file or buffer contents do not match the requested format */

/* Read a CSR matrix from `path` (FB_FILE_MTX general or symmetric, FB_FILE_CSR,
 * FB_FILE_BINARY). The arrays of *out are allocated by the library; free them with
 * fb_io_csr_release. The result can be handed to fb_mg_create_csr as is.
 * Replaces SparseMatrixCSR::read_from (kernel/lafem/sparse_matrix_csr.hpp:1098-1246). */
FB_API int fb_io_csr_read(const char* path, int mode, fb_csr_host* out);
/* Write a CSR matrix (FB_FILE_MTX, FB_FILE_CSR, FB_FILE_BINARY); symmetric != 0 writes the
 * lower triangle as "coordinate real symmetric" (FB_FILE_MTX only), byte for byte as
 * SparseMatrixCSR::write_out (sparse_matrix_csr.hpp:1261-1343). */
FB_API int fb_io_csr_write(const char* path, int mode, const fb_csr_host* m, int symmetric);
/* In-memory serialisation in the fm_csr layout (SparseMatrixCSR::serialise/deserialise,
 * sparse_matrix_csr.hpp:1066-1090; Container::_serialise, container.hpp:317-572). */
FB_API int fb_io_csr_serialised_size(const fb_csr_host* m, uint64_t* size);
FB_API int fb_io_csr_serialise(const fb_csr_host* m, void* buf, uint64_t capacity);
FB_API int fb_io_csr_deserialise(const void* buf, uint64_t size, fb_csr_host* out);
FB_API void fb_io_csr_release(fb_csr_host* m);

/* Read / write a dense vector (FB_FILE_EXP, FB_FILE_MTX, FB_FILE_DV, FB_FILE_BINARY); *data
 * is allocated by the library, free it with fb_io_free. Replaces DenseVector::read_from /
 * write_out / serialise / deserialise (kernel/lafem/dense_vector.hpp:480-505, 587-777). */
FB_API int fb_io_vector_read(const char* path, int mode, uint64_t* n, double** data);
FB_API int fb_io_vector_write(const char* path, int mode, const double* data, uint64_t n);
FB_API int fb_io_vector_serialised_size(uint64_t n, uint64_t* size);
FB_API int fb_io_vector_serialise(const double* data, uint64_t n, void* buf, uint64_t capacity);
FB_API int fb_io_vector_deserialise(const void* buf, uint64_t size, uint64_t* n, double** data);
/* Read / write a sparse vector as MatrixMarket "coordinate real general" with one column
 * (FB_FILE_MTX only, as the reference), e.g. a UnitFilter's Dirichlet list
 * (UnitFilter::get_filter_vector().write_out(fm_mtx, ...)). Read: indices 0-based, sorted, a
 * repeated index keeps its last value; *indices and *values are freed with fb_io_free. Write:
 * indices strictly ascending and < size. Replaces SparseVector::read_from / write_out
 * (kernel/lafem/sparse_vector.hpp:517-680). */
FB_API int fb_io_sparse_vector_read(const char* path, int mode, uint64_t* size, uint64_t* nnz, uint64_t** indices,
                                    double** values);
FB_API int fb_io_sparse_vector_write(const char* path, int mode, uint64_t size, uint64_t nnz, const uint64_t* indices,
                                     const double* values);
FB_API void fb_io_free(void* p);

/* library version string */
FB_API const char* fb_version(void);

#ifdef __cplusplus
}
#endif
#endif /* FEAT3_B200_H */
