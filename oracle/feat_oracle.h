/*
 * CPU oracle for the FEAT3 geometric-multigrid Poisson hot path.
 *
 * TEST INFRASTRUCTURE ONLY: this library is the checker used by tests/, by
 * __graft_entry__.smoke() and by bench.py's CPU-baseline leg. Nothing in the product
 * (feat3_b200/) may load or call it.
 *
 * It restates, in plain C++, the reference algorithms on structured unit-square /
 * unit-cube hierarchies with lexicographic numbering (loops whose iterations are
 * independent run on OpenMP threads and compute what the serial loop computes; the
 * reductions are sequential, in the reference's order):
 *   - Q1/Q2 Laplace assembly with 3-point Gauss-Legendre per direction
 *       (kernel/assembly/bilinear_operator_assembler.hpp:218-339,
 *        kernel/assembly/common_operators.hpp:36-97, cubature "auto-degree:5")
 *   - load vectors for f = d*pi^2*prod(sin(pi x_i)), f = 1, and the exp-bubble
 *       (kernel/assembly/common_functionals.hpp:137-225, kernel/analytic/common.hpp)
 *   - homogeneous Dirichlet unit filter (kernel/lafem/unit_filter.hpp:399-437)
 *   - nested-space prolongation P and R = P^T
 *       (kernel/assembly/grid_transfer.hpp:304-321, tutorial_05_multigrid.cpp:302)
 *   - CSR apply r = b*y + a*A*x (kernel/lafem/arch/apply_generic.hpp:25-70)
 *   - Jacobi / Richardson smoother, V-cycle, PCG, Richardson outer solver
 *       (kernel/solver/{jacobi_precond,richardson,multigrid,pcg,iterative}.hpp)
 *   - mixed precision by conversion (kernel/solver/convert_precond.hpp:41-120)
 *   - the adjoint element gradient dJ/dk_e = -lambda_e^T K_e u_e
 * Parity of this restatement is pinned against the reference's own solver
 * (oracle/_ref/feat_ref, built from the reference sources) through the fixtures in
 * tests/golden/.
 */
#ifndef FEAT3_ORACLE_H
#define FEAT3_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

typedef struct or_hier or_hier;

/* hierarchy of structured levels level_min..level; kfine: per-element coefficient on the
 * finest level (lexicographic, N^dim values) or NULL for k = 1; coarse k = mean of children */
or_hier* or_hier_create(int dim, int degree, int level, int level_min, const double* kfine);
void or_hier_destroy(or_hier* h);

int64_t or_level_ndofs(const or_hier* h, int level);
int64_t or_level_nnz(const or_hier* h, int level);
/* CSR of A on a level: rowptr[n+1], col[nnz], val[nnz] */
void or_level_csr(const or_hier* h, int level, int64_t* rowptr, int32_t* col, double* val);
/* prolongation from level-1 to level (rows = fine dofs) and its transpose */
int64_t or_level_pnnz(const or_hier* h, int level);
void or_level_p(const or_hier* h, int level, int64_t* rowptr, int32_t* col, double* val);
void or_level_r(const or_hier* h, int level, int64_t* rowptr, int32_t* col, double* val);
int64_t or_level_nfilter(const or_hier* h, int level);
void or_level_filter(const or_hier* h, int level, int32_t* idx);
/* unit-coefficient element stiffness matrix (row-major, nloc x nloc) on a level */
int or_element_matrix(const or_hier* h, int level, double* kref);

/* load vector on the finest level: kind 0 = sine bubble, 1 = one, 2 = exp bubble; filtered */
void or_rhs(const or_hier* h, int kind, double* rhs);

typedef struct or_cfg {
  int solver;        /* 0 = PCG, 1 = Richardson */
  int nu;            /* smoothing steps (pre = post) */
  double omega_jac;  /* Jacobi damping */
  double omega_rich; /* Richardson smoother damping */
  double omega_outer;/* outer Richardson damping */
  int coarse;        /* 0 = direct, 1 = PCG (default settings), 2 = smoother, 3 = none */
  double tol_rel;
  int max_iter;
  int inner;         /* 0 = FP64 multigrid, 1 = FP32 multigrid, 2 = FP32 with FP16-quantised matrices */
  int cycle;         /* 0 = V, 1 = F, 2 = W (Solver::MultiGridCycle) */
  int cgc;           /* 0 = fixed, 1 = min-energy, 2 = min-defect (Solver::MultiGridAdaptCGC) */
} or_cfg;

/* solves A sol = rhs with the configured solver (sol holds the initial guess).
 * hist receives the defect norms (max_iter + 1 entries), iters the iteration count.
 * Returns the reference Status code (0 undefined, 1 progress, 2 success, 3 aborted,
 * 4 diverged, 5 max_iter, 6 stagnated). */
int or_solve(const or_hier* h, const or_cfg* cfg, const double* rhs, double* sol, double* hist, int* iters);

/* one multigrid cycle of the configured type (preconditioner application): cor = MG(def) */
void or_vcycle(const or_hier* h, const or_cfg* cfg, const double* def, double* cor);

/* element gradient on the finest level: grad[e] = -lambda_e^T K_e^(1) u_e */
void or_element_grad(const or_hier* h, const double* u, const double* lam, double* grad);

/* r = b*y + a*A*x for an explicit CSR matrix (apply_generic.hpp:25-70), transposed optional */
void or_csr_apply(double* r, double a, const double* x, double b, const double* y,
                  const double* val, const int32_t* col, const int64_t* rowptr,
                  int64_t rows, int64_t cols, int transposed);

/* FEAT3's numbering of the unit square / cube refined `level` times
 * (RefinedUnitCubeFactory = UnitCubeFactory + StandardRefinery, common_factories.hpp:71-235,
 * conformal_mesh.hpp:439-528): dof_lex[f] = lexicographic lattice index of FEAT DOF f of the
 * Q1 (degree 1) or Q2 (degree 2) space, cell_lex[c] = lexicographic index of FEAT cell c.
 * Either pointer may be NULL. Returns 0, or -1 for unsupported arguments. */
int or_feat_numbering(int dim, int degree, int level, uint32_t* dof_lex, uint32_t* cell_lex);

/* threads of the parallel loops (OpenMP), 1 when built without OpenMP */
int or_threads(void);

#ifdef __cplusplus
}
#endif
#endif
