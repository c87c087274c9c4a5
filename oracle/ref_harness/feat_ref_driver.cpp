// Oracle-side driver that runs the REFERENCE's own CPU solver (FEAT3, built from its
// sources by oracle/Makefile) on the structured Poisson configurations this project
// measures, and dumps its results for the parity tests.
//
// This file is TEST INFRASTRUCTURE. It is compiled against the reference headers
// (kernel/solver/multigrid.hpp, pcg.hpp, richardson.hpp, jacobi_precond.hpp,
// convert_precond.hpp, kernel/assembly/*) and never linked into the product.
//
// What it adds on top of the reference (the reference itself is untouched):
//   * a per-element diffusion coefficient operator (the Laplace operator of
//     kernel/assembly/common_operators.hpp:36-97 scaled by k[cell], read through
//     trafo_eval.get_cell_index(), kernel/trafo/evaluator_base.hpp:189);
//   * a dense direct coarse-grid solver (UMFPACK is not available offline);
//   * FP16-storage emulation of the inner multigrid matrices (quantise/dequantise);
//   * the FP64 adjoint gradient dJ/dk_e = -int_e grad(lambda).grad(u).
//
// Structured input fields (coefficient k per element, target vectors) are passed in
// lexicographic lattice order and mapped to FEAT cells / DOFs through centroids and
// DOF coordinates, so the numbering of the reference's refined meshes never has to be
// reproduced.
#include <kernel/util/runtime.hpp>
#include <kernel/util/string.hpp>
#include <kernel/util/time_stamp.hpp>
#include <kernel/geometry/boundary_factory.hpp>
#include <kernel/geometry/conformal_mesh.hpp>
#include <kernel/geometry/common_factories.hpp>
#include <kernel/geometry/mesh_part.hpp>
#include <kernel/trafo/standard/mapping.hpp>
#include <kernel/space/lagrange1/element.hpp>
#include <kernel/space/lagrange2/element.hpp>
#include <kernel/cubature/dynamic_factory.hpp>
#include <kernel/analytic/common.hpp>
#include <kernel/analytic/static_wrapper.hpp>
#include <kernel/assembly/symbolic_assembler.hpp>
#include <kernel/assembly/unit_filter_assembler.hpp>
#include <kernel/assembly/bilinear_operator_assembler.hpp>
#include <kernel/assembly/linear_functional_assembler.hpp>
#include <kernel/assembly/common_operators.hpp>
#include <kernel/assembly/common_functionals.hpp>
#include <kernel/assembly/grid_transfer.hpp>
#include <kernel/assembly/interpolator.hpp>
#include <kernel/assembly/asm_traits.hpp>
#include <kernel/lafem/dense_vector.hpp>
#include <kernel/lafem/sparse_matrix_csr.hpp>
#include <kernel/lafem/unit_filter.hpp>
#include <kernel/lafem/transfer.hpp>
#include <kernel/solver/multigrid.hpp>
#include <kernel/solver/pcg.hpp>
#include <kernel/solver/richardson.hpp>
#include <kernel/solver/jacobi_precond.hpp>
#include <kernel/solver/convert_precond.hpp>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cmath>
#include <deque>
#include <memory>
#include <vector>
#include <string>
#include <fstream>
#include <iostream>
#include <algorithm>

using namespace FEAT;

namespace RefDriver
{
  struct Config
  {
    int dim = 2;           // 2 or 3
    int degree = 1;        // 1 = Q1, 2 = Q2
    int level = 4;         // finest level: N = 2^level cells per side
    int level_min = 1;     // coarsest level
    std::string rhs = "sine";      // sine | one | expbubble
    std::string kfile;             // per-element k on the finest level (lexicographic), optional
    std::string solver = "pcg";    // pcg | richardson
    int nu = 4;                    // pre = post smoothing steps
    double omega_jac = 0.5;        // Jacobi damping (inside Richardson)
    double omega_rich = 1.0;       // Richardson smoother damping
    double omega_outer = 1.0;      // outer Richardson damping
    std::string coarse = "direct"; // direct | pcg | smoother | none
    double tol = 1e-8;
    int maxit = 1000;
    std::string inner = "f64";     // f64 | f32 | f16 (mixed: FP64 outer, ConvertPrecond to FP32 MG)
    std::string cycle = "v";       // v | f | w (Solver::MultiGridCycle)
    std::string cgc = "fixed";     // fixed | energy | defect (Solver::MultiGridAdaptCGC)
    std::string target;            // adjoint: u_target in lexicographic DOF lattice order
    std::string out = "ref";
    bool dump_matrices = false;
    bool feat_files = false;       // also write the hierarchy through the reference's own write_out
    bool quiet = false;
    int repeat = 1;                // timed solves (each from a zero initial guess)
    double budget_s = 0.0;         // > 0: no further timed solve once the next would end past this
    int warmup = 0;                // untimed solves of one iteration each before the timed ones
  };

  // ---------------------------------------------------------------------------------------
  // small binary I/O helpers
  static void write_f64(const std::string& fn, const std::vector<double>& v)
  {
    FILE* f = std::fopen(fn.c_str(), "wb");
    if(!f) { std::cerr << "cannot write " << fn << std::endl; std::exit(2); }
    if(!v.empty()) std::fwrite(v.data(), sizeof(double), v.size(), f);
    std::fclose(f);
  }
  static void write_u64(const std::string& fn, const std::vector<unsigned long>& v)
  {
    FILE* f = std::fopen(fn.c_str(), "wb");
    if(!f) { std::cerr << "cannot write " << fn << std::endl; std::exit(2); }
    if(!v.empty()) std::fwrite(v.data(), sizeof(unsigned long), v.size(), f);
    std::fclose(f);
  }
  static std::vector<double> read_f64(const std::string& fn)
  {
    std::vector<double> v;
    FILE* f = std::fopen(fn.c_str(), "rb");
    if(!f) { std::cerr << "cannot read " << fn << std::endl; std::exit(2); }
    std::fseek(f, 0, SEEK_END);
    long sz = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    v.resize(std::size_t(sz) / sizeof(double));
    if(!v.empty() && std::fread(v.data(), sizeof(double), v.size(), f) != v.size())
    {
      std::cerr << "short read " << fn << std::endl; std::exit(2);
    }
    std::fclose(f);
    return v;
  }

  // ---------------------------------------------------------------------------------------
  // coordinate functions for DOF-coordinate interpolation (Lagrange node functionals are
  // point evaluations, so interpolating x/y/z yields the DOF node coordinates)
  template<typename DT_, int c_>
  class CoordStatic
  {
  public:
    static DT_ eval(DT_ x) { return x; }
    static DT_ eval(DT_ x, DT_ y) { return c_ == 0 ? x : y; }
    static DT_ eval(DT_ x, DT_ y, DT_ z) { return c_ == 0 ? x : (c_ == 1 ? y : z); }
  };
  template<typename DT_> using CoordX = CoordStatic<DT_, 0>;
  template<typename DT_> using CoordY = CoordStatic<DT_, 1>;
  template<typename DT_> using CoordZ = CoordStatic<DT_, 2>;

  // constant-one right-hand side  f = 1
  template<typename DT_>
  class OneStatic
  {
  public:
    static DT_ eval(DT_) { return DT_(1); }
    static DT_ eval(DT_, DT_) { return DT_(1); }
    static DT_ eval(DT_, DT_, DT_) { return DT_(1); }
  };

  // ---------------------------------------------------------------------------------------
  // Laplace operator with a piecewise-constant coefficient per cell
  class CoefLaplaceOperator :
    public Assembly::BilinearOperator
  {
  public:
    static constexpr TrafoTags trafo_config = TrafoTags::none;
    static constexpr SpaceTags test_config = SpaceTags::grad;
    static constexpr SpaceTags trial_config = SpaceTags::grad;

    const std::vector<double>* kcell;
    explicit CoefLaplaceOperator(const std::vector<double>* k) : kcell(k) {}

    template<typename AsmTraits_>
    class Evaluator :
      public Assembly::BilinearOperator::Evaluator<AsmTraits_>
    {
    public:
      typedef typename AsmTraits_::DataType DataType;
      typedef typename AsmTraits_::TrafoEvaluator TrafoEvaluator;
      typedef typename AsmTraits_::TrialBasisData TrialBasisData;
      typedef typename AsmTraits_::TestBasisData TestBasisData;
    protected:
      const std::vector<double>& _k;
      DataType _kc;
    public:
      explicit Evaluator(const CoefLaplaceOperator& op) : _k(*op.kcell), _kc(1) {}
      void prepare(const TrafoEvaluator& trafo_eval)
      {
        _kc = DataType(_k.at(trafo_eval.get_cell_index()));
      }
      DataType operator()(const TrialBasisData& phi, const TestBasisData& psi)
      {
        return _kc * dot(phi.grad, psi.grad);
      }
    };
  };

  // ---------------------------------------------------------------------------------------
  // dense direct coarse-grid solver on the filtered coarse matrix (LU, partial pivoting)
  template<typename Matrix_, typename Filter_>
  class DenseDirectSolver :
    public Solver::SolverBase<typename Matrix_::VectorTypeL>
  {
  public:
    typedef typename Matrix_::VectorTypeL VectorType;
    typedef typename Matrix_::DataType DataType;
  protected:
    const Matrix_& _matrix;
    const Filter_& _filter;
    Index _n;
    std::vector<double> _lu;
    std::vector<Index> _piv;
  public:
    DenseDirectSolver(const Matrix_& matrix, const Filter_& filter) : _matrix(matrix), _filter(filter), _n(0) {}
    virtual String name() const override { return "DenseDirect"; }
    virtual void init_numeric() override
    {
      _n = _matrix.rows();
      const Index n = _n;
      _lu.assign(n*n, 0.0);
      const auto* rp = _matrix.row_ptr();
      const auto* ci = _matrix.col_ind();
      const auto* va = _matrix.val();
      std::vector<char> dir(n, 0);
      for(Index i(0); i < _filter.used_elements(); ++i)
        dir[_filter.get_indices()[i]] = 1;
      for(Index i(0); i < n; ++i)
      {
        if(dir[i]) { _lu[i*n+i] = 1.0; continue; }
        for(auto j = rp[i]; j < rp[i+1]; ++j)
          if(!dir[ci[j]]) _lu[i*n + ci[j]] = double(va[j]);
      }
      _piv.resize(n);
      for(Index k(0); k < n; ++k)
      {
        Index p = k;
        for(Index i(k+1); i < n; ++i)
          if(std::fabs(_lu[i*n+k]) > std::fabs(_lu[p*n+k])) p = i;
        _piv[k] = p;
        if(p != k) for(Index j(0); j < n; ++j) std::swap(_lu[k*n+j], _lu[p*n+j]);
        const double d = _lu[k*n+k];
        for(Index i(k+1); i < n; ++i)
        {
          const double l = (_lu[i*n+k] /= d);
          for(Index j(k+1); j < n; ++j) _lu[i*n+j] -= l * _lu[k*n+j];
        }
      }
    }
    virtual Solver::Status apply(VectorType& vec_cor, const VectorType& vec_def) override
    {
      const Index n = _n;
      std::vector<double> b(n);
      for(Index i(0); i < n; ++i) b[i] = double(vec_def(i));
      for(Index i(0); i < _filter.used_elements(); ++i) b[_filter.get_indices()[i]] = 0.0;
      for(Index k(0); k < n; ++k) if(_piv[k] != k) std::swap(b[k], b[_piv[k]]);
      for(Index i(0); i < n; ++i) for(Index j(0); j < i; ++j) b[i] -= _lu[i*n+j] * b[j];
      for(Index i(n); i > 0; --i)
      {
        const Index r = i-1;
        for(Index j(r+1); j < n; ++j) b[r] -= _lu[r*n+j] * b[j];
        b[r] /= _lu[r*n+r];
      }
      for(Index i(0); i < n; ++i) vec_cor(i, DataType(b[i]));
      _filter.filter_cor(vec_cor);
      return Solver::Status::success;
    }
  };

  // ---------------------------------------------------------------------------------------
  // PCG / Richardson that record every defect norm they compute (full precision)
  template<typename Matrix_, typename Filter_>
  class RecPCG : public Solver::PCG<Matrix_, Filter_>
  {
  public:
    typedef Solver::PCG<Matrix_, Filter_> Base;
    typedef typename Base::VectorType VectorType;
    typedef typename Base::PrecondType PrecondType;
    std::vector<double> hist;
    RecPCG(const Matrix_& m, const Filter_& f, std::shared_ptr<PrecondType> p) : Base(m, f, p) {}
  protected:
    virtual Solver::Status _set_initial_defect(const VectorType& d, const VectorType& s) override
    {
      auto st = Base::_set_initial_defect(d, s); hist.clear(); hist.push_back(double(this->_def_cur)); return st;
    }
    virtual Solver::Status _set_new_defect(const VectorType& d, const VectorType& s) override
    {
      auto st = Base::_set_new_defect(d, s); hist.push_back(double(this->_def_cur)); return st;
    }
  };
  template<typename Matrix_, typename Filter_>
  class RecRichardson : public Solver::Richardson<Matrix_, Filter_>
  {
  public:
    typedef Solver::Richardson<Matrix_, Filter_> Base;
    typedef typename Base::VectorType VectorType;
    typedef typename Base::PrecondType PrecondType;
    std::vector<double> hist;
    RecRichardson(const Matrix_& m, const Filter_& f, double w, std::shared_ptr<PrecondType> p) : Base(m, f, typename Matrix_::DataType(w), p) {}
  protected:
    virtual Solver::Status _set_initial_defect(const VectorType& d, const VectorType& s) override
    {
      auto st = Base::_set_initial_defect(d, s); hist.clear(); hist.push_back(double(this->_def_cur)); return st;
    }
    virtual Solver::Status _set_new_defect(const VectorType& d, const VectorType& s) override
    {
      auto st = Base::_set_new_defect(d, s); hist.push_back(double(this->_def_cur)); return st;
    }
  };

  // ---------------------------------------------------------------------------------------
  template<typename Shape_, template<typename> class Element_>
  class Runner
  {
  public:
    typedef Shape_ ShapeType;
    static constexpr int dim = ShapeType::dimension;
    typedef Geometry::ConformalMesh<ShapeType> MeshType;
    typedef Geometry::MeshPart<MeshType> MeshPartType;
    typedef Trafo::Standard::Mapping<MeshType> TrafoType;
    typedef Element_<TrafoType> SpaceType;
    typedef LAFEM::DenseVector<Mem::Main, double, Index> VectorType;
    typedef LAFEM::SparseMatrixCSR<Mem::Main, double, Index> MatrixType;
    typedef LAFEM::UnitFilter<Mem::Main, double, Index> FilterType;
    typedef LAFEM::Transfer<MatrixType> TransferType;
    typedef LAFEM::DenseVector<Mem::Main, float, Index> VectorTypeF;
    typedef LAFEM::SparseMatrixCSR<Mem::Main, float, Index> MatrixTypeF;
    typedef LAFEM::UnitFilter<Mem::Main, float, Index> FilterTypeF;
    typedef LAFEM::Transfer<MatrixTypeF> TransferTypeF;

    struct Level
    {
      MeshType mesh;
      TrafoType trafo;
      SpaceType space;
      MatrixType matrix;
      FilterType filter;
      TransferType transfer;
      MatrixTypeF matrix_f;
      FilterTypeF filter_f;
      TransferTypeF transfer_f;
      int lvl;
      std::vector<double> kcell;   // coefficient per FEAT cell
      explicit Level(Geometry::Factory<MeshType>& fac) : mesh(fac), trafo(mesh), space(trafo), lvl(0) {}
    };

    const Config& cfg;
    std::deque<std::shared_ptr<Level>> levels; // front = finest
    std::ofstream info;
    std::vector<double> solve_times;           // every timed solve of the run

    explicit Runner(const Config& c) : cfg(c) {}

    // lexicographic cell index of a FEAT cell (through its centroid) on a level with N cells per side
    Index cell_lex(const MeshType& mesh, Index cell, Index N) const
    {
      const auto& iset = mesh.template get_index_set<dim, 0>();
      const auto& vtx = mesh.get_vertex_set();
      double c[3] = {0.0, 0.0, 0.0};
      const int nv = iset.num_indices;
      for(int j(0); j < nv; ++j)
        for(int d(0); d < dim; ++d)
          c[d] += double(vtx[iset(cell, j)][d]);
      Index idx = 0, stride = 1;
      for(int d(0); d < dim; ++d)
      {
        double x = c[d] / double(nv);
        Index ix = Index(std::floor(x * double(N)));
        if(ix >= N) ix = N-1;
        idx += ix * stride;
        stride *= N;
      }
      return idx;
    }

    // DOF node coordinates via interpolation of the coordinate functions
    std::vector<double> dof_coords(const Level& lv) const
    {
      const Index n = lv.space.get_num_dofs();
      std::vector<double> xyz(n * dim);
      VectorType v(n);
      for(int d(0); d < dim; ++d)
      {
        if(d == 0) { Analytic::StaticWrapperFunction<dim, CoordX, true, false, false> f; Assembly::Interpolator::project(v, f, lv.space); }
        if(d == 1) { Analytic::StaticWrapperFunction<dim, CoordY, true, false, false> f; Assembly::Interpolator::project(v, f, lv.space); }
        if(d == 2) { Analytic::StaticWrapperFunction<dim, CoordZ, true, false, false> f; Assembly::Interpolator::project(v, f, lv.space); }
        for(Index i(0); i < n; ++i) xyz[i*dim + d] = v(i);
      }
      return xyz;
    }

    // lexicographic lattice index of each DOF (lattice of (degree*N+1)^dim points)
    std::vector<Index> dof_lattice(const Level& lv, Index N) const
    {
      const auto xyz = dof_coords(lv);
      const Index M = Index(cfg.degree) * N;
      const Index n = lv.space.get_num_dofs();
      std::vector<Index> lat(n);
      for(Index i(0); i < n; ++i)
      {
        Index idx = 0, stride = 1;
        for(int d(0); d < dim; ++d)
        {
          Index ix = Index(std::llround(xyz[i*dim + d] * double(M)));
          idx += ix * stride;
          stride *= (M + 1);
        }
        lat[i] = idx;
      }
      return lat;
    }

    void dump_csr(const std::string& pre, const MatrixType& a) const
    {
      std::vector<unsigned long> rp(a.row_ptr(), a.row_ptr() + a.rows() + 1);
      std::vector<unsigned long> ci(a.col_ind(), a.col_ind() + a.used_elements());
      std::vector<double> va(a.val(), a.val() + a.used_elements());
      write_u64(pre + ".rowptr", rp);
      write_u64(pre + ".col", ci);
      write_f64(pre + ".val", va);
    }

    // The hierarchy in the reference's own container file formats (SparseMatrixCSR::write_out,
    // kernel/lafem/sparse_matrix_csr.hpp:1261-1343), plus the reference's parse of its own
    // text files written back in binary form (read_from, sparse_matrix_csr.hpp:1098-1246),
    // so both directions of the I/O layer can be checked against the reference.
    void write_feat_files(const std::string& pre, const Level& lv, bool transfers) const
    {
      lv.matrix.write_out(LAFEM::FileMode::fm_csr, pre + ".A.csr");
      lv.matrix.write_out(LAFEM::FileMode::fm_mtx, pre + ".A.mtx");
      lv.matrix.write_out(LAFEM::FileMode::fm_mtx, pre + ".A.sym.mtx", true);
      for(const char* nm : {".A.mtx", ".A.sym.mtx"})
      {
        MatrixType back;
        back.read_from(LAFEM::FileMode::fm_mtx, pre + nm);
        back.write_out(LAFEM::FileMode::fm_csr, pre + nm + ".csr");
      }
      MatrixType bin;
      bin.read_from(LAFEM::FileMode::fm_binary, pre + ".A.csr");
      bin.write_out(LAFEM::FileMode::fm_binary, pre + ".A.csr.csr");
      // the Dirichlet filter's sparse vector (SparseVector::write_out / read_from,
      // kernel/lafem/sparse_vector.hpp:517-680)
      lv.filter.get_filter_vector().write_out(LAFEM::FileMode::fm_mtx, pre + ".filter.mtx");
      LAFEM::SparseVector<Mem::Main, double, Index> fv;
      fv.read_from(LAFEM::FileMode::fm_mtx, pre + ".filter.mtx");
      fv.write_out(LAFEM::FileMode::fm_mtx, pre + ".filter.mtx.mtx");
      if(transfers)
      {
        lv.transfer.get_mat_prol().write_out(LAFEM::FileMode::fm_csr, pre + ".P.csr");
        lv.transfer.get_mat_prol().write_out(LAFEM::FileMode::fm_mtx, pre + ".P.mtx");
        lv.transfer.get_mat_rest().write_out(LAFEM::FileMode::fm_csr, pre + ".R.csr");
        lv.transfer.get_mat_rest().write_out(LAFEM::FileMode::fm_mtx, pre + ".R.mtx");
      }
    }

    // DenseVector::write_out / read_from (kernel/lafem/dense_vector.hpp:587-777)
    static void write_feat_vector(const std::string& pre, const VectorType& v)
    {
      v.write_out(LAFEM::FileMode::fm_dv, pre + ".dv");
      v.write_out(LAFEM::FileMode::fm_exp, pre + ".exp");
      v.write_out(LAFEM::FileMode::fm_mtx, pre + ".vmtx");
      VectorType a, b;
      a.read_from(LAFEM::FileMode::fm_exp, pre + ".exp");
      a.write_out(LAFEM::FileMode::fm_dv, pre + ".exp.dv");
      b.read_from(LAFEM::FileMode::fm_mtx, pre + ".vmtx");
      b.write_out(LAFEM::FileMode::fm_dv, pre + ".vmtx.dv");
    }

    int run()
    {
      info.open(cfg.out + ".info");
      info.precision(17);
      TimeStamp stamp_setup;

      // ---- mesh hierarchy (tutorials/tutorial_05_multigrid.cpp:173-216)
      {
        Geometry::RefinedUnitCubeFactory<MeshType> fac(Index(cfg.level_min));
        levels.push_front(std::make_shared<Level>(fac));
        levels.front()->lvl = cfg.level_min;
      }
      for(int l = cfg.level_min; l < cfg.level; ++l)
      {
        Geometry::StandardRefinery<MeshType> fac(levels.front()->mesh);
        levels.push_front(std::make_shared<Level>(fac));
        levels.front()->lvl = l + 1;
      }

      // ---- coefficient fields per level (lexicographic on the finest level, coarse = mean of children)
      std::vector<std::vector<double>> klex(cfg.level + 1);
      const bool have_k = !cfg.kfile.empty();
      if(have_k)
      {
        klex[cfg.level] = read_f64(cfg.kfile);
        Index Nf = Index(1) << cfg.level;
        Index ne = 1; for(int d(0); d < dim; ++d) ne *= Nf;
        if(klex[cfg.level].size() != ne) { std::cerr << "kfile size mismatch" << std::endl; return 2; }
        for(int l = cfg.level - 1; l >= cfg.level_min; --l)
        {
          const Index Nc = Index(1) << l, Nfl = Nc * 2;
          Index nec = 1; for(int d(0); d < dim; ++d) nec *= Nc;
          klex[l].assign(nec, 0.0);
          for(Index e(0); e < nec; ++e)
          {
            Index cx = e % Nc, cy = (e / Nc) % Nc, cz = (dim == 3) ? e / (Nc*Nc) : 0;
            double s = 0.0;
            for(int c(0); c < (1 << dim); ++c)
            {
              Index fx = 2*cx + (c & 1), fy = 2*cy + ((c >> 1) & 1), fz = (dim == 3) ? 2*cz + ((c >> 2) & 1) : 0;
              s += klex[l+1][fx + Nfl*(fy + Nfl*fz)];
            }
            klex[l][e] = s / double(1 << dim);
          }
        }
      }

      Cubature::DynamicFactory cubature("auto-degree:5");

      // ---- matrices and filters (tutorial_05_multigrid.cpp:226-250)
      for(auto& lp : levels)
      {
        Level& lv = *lp;
        const Index N = Index(1) << lv.lvl;
        Assembly::SymbolicAssembler::assemble_matrix_std1(lv.matrix, lv.space);
        lv.matrix.format();
        if(have_k)
        {
          const Index nc = lv.mesh.get_num_elements();
          lv.kcell.resize(nc);
          for(Index c(0); c < nc; ++c) lv.kcell[c] = klex[lv.lvl][cell_lex(lv.mesh, c, N)];
          CoefLaplaceOperator op(&lv.kcell);
          Assembly::BilinearOperatorAssembler::assemble_matrix1(lv.matrix, op, lv.space, cubature);
        }
        else
        {
          Assembly::Common::LaplaceOperator op;
          Assembly::BilinearOperatorAssembler::assemble_matrix1(lv.matrix, op, lv.space, cubature);
        }
        Geometry::BoundaryFactory<MeshType> bnd_fac(lv.mesh);
        MeshPartType boundary(bnd_fac);
        Assembly::UnitFilterAssembler<MeshType> unit_asm;
        unit_asm.add_mesh_part(boundary);
        unit_asm.assemble(lv.filter, lv.space);
      }

      // ---- grid transfers (tutorial_05_multigrid.cpp:263-303)
      for(std::size_t i(0); i + 1 < levels.size(); ++i)
      {
        Level& lf = *levels.at(i);
        Level& lc = *levels.at(i+1);
        MatrixType& p = lf.transfer.get_mat_prol();
        Assembly::SymbolicAssembler::assemble_matrix_2lvl(p, lf.space, lc.space);
        p.format();
        Assembly::GridTransfer::assemble_prolongation_direct(p, lf.space, lc.space, cubature);
        lf.transfer.get_mat_rest() = p.transpose();
      }

      // ---- fine-level vectors (tutorial_05_multigrid.cpp:315-341)
      Level& top = *levels.front();
      VectorType vec_sol = top.matrix.create_vector_r();
      VectorType vec_rhs = top.matrix.create_vector_r();
      vec_sol.format();
      vec_rhs.format();
      if(cfg.rhs == "sine")
      {
        Analytic::Common::SineBubbleFunction<dim> sol_function;
        Assembly::Common::LaplaceFunctional<decltype(sol_function)> force(sol_function);
        Assembly::LinearFunctionalAssembler::assemble_vector(vec_rhs, force, top.space, cubature);
      }
      else if(cfg.rhs == "expbubble")
      {
        Analytic::Common::ExpBubbleFunction<dim> sol_function;
        Assembly::Common::LaplaceFunctional<decltype(sol_function)> force(sol_function);
        Assembly::LinearFunctionalAssembler::assemble_vector(vec_rhs, force, top.space, cubature);
      }
      else
      {
        Analytic::StaticWrapperFunction<dim, OneStatic, true, false, false> one;
        Assembly::Common::ForceFunctional<decltype(one)> force(one);
        Assembly::LinearFunctionalAssembler::assemble_vector(vec_rhs, force, top.space, cubature);
      }
      top.filter.filter_sol(vec_sol);
      top.filter.filter_rhs(vec_rhs);

      const double setup_time = stamp_setup.elapsed_now();

      // ---- dumps of the hierarchy (for drop-in operator parity tests)
      {
        const Index Nt = Index(1) << top.lvl;
        const auto lat = dof_lattice(top, Nt);
        std::vector<unsigned long> latv(lat.begin(), lat.end());
        write_u64(cfg.out + ".lattice", latv);
        write_f64(cfg.out + ".coords", dof_coords(top));
        write_f64(cfg.out + ".rhs", std::vector<double>(vec_rhs.elements(), vec_rhs.elements() + vec_rhs.size()));
      }
      if(cfg.dump_matrices)
      {
        for(std::size_t i(0); i < levels.size(); ++i)
        {
          Level& lv = *levels.at(i);
          const std::string pre = cfg.out + ".L" + std::to_string(lv.lvl);
          dump_csr(pre + ".A", lv.matrix);
          std::vector<unsigned long> fi(lv.filter.get_indices(), lv.filter.get_indices() + lv.filter.used_elements());
          write_u64(pre + ".filter", fi);
          const Index N = Index(1) << lv.lvl;
          const auto lat = dof_lattice(lv, N);
          write_u64(pre + ".lattice", std::vector<unsigned long>(lat.begin(), lat.end()));
          // lexicographic index of each of the level's cells, in FEAT's cell numbering
          std::vector<unsigned long> cells(lv.mesh.get_num_elements());
          for(Index c(0); c < lv.mesh.get_num_elements(); ++c)
            cells[c] = cell_lex(lv.mesh, c, N);
          write_u64(pre + ".cells", cells);
          if(i + 1 < levels.size())
          {
            dump_csr(pre + ".P", lv.transfer.get_mat_prol());
            dump_csr(pre + ".R", lv.transfer.get_mat_rest());
          }
          if(cfg.feat_files)
            write_feat_files(pre, lv, i + 1 < levels.size());
        }
        if(cfg.feat_files)
          write_feat_vector(cfg.out + ".rhs", vec_rhs);
      }

      // ---- solve
      std::vector<double> hist;
      int iters = 0;
      int status = 0;
      double solve_time = 0.0;
      bool mixed = (cfg.inner != "f64");
      if(!mixed)
        solve_f64(vec_sol, vec_rhs, hist, iters, status, solve_time);
      else
        solve_mixed(vec_sol, vec_rhs, hist, iters, status, solve_time);

      write_f64(cfg.out + ".u", std::vector<double>(vec_sol.elements(), vec_sol.elements() + vec_sol.size()));
      if(cfg.feat_files)
        vec_sol.write_out(LAFEM::FileMode::fm_dv, cfg.out + ".u.dv");

      info << "n_dofs " << top.space.get_num_dofs() << "\n";
      info << "n_cells " << top.mesh.get_num_elements() << "\n";
      info << "nnz " << top.matrix.used_elements() << "\n";
      info << "iters " << iters << "\n";
      info << "status " << status << "\n";
      info << "solve_time " << solve_time << "\n";
      info << "setup_time " << setup_time << "\n";
      info << "warmup_solves " << cfg.warmup << "\n";
      info << "solve_times";
      for(double st : solve_times) info << " " << st;
      info << "\n";
      info << "def_init " << (hist.empty() ? 0.0 : hist.front()) << "\n";
      info << "def_final " << (hist.empty() ? 0.0 : hist.back()) << "\n";
      info << "hist";
      for(double h : hist) info << " " << h;
      info << "\n";

      // ---- adjoint gradient
      if(!cfg.target.empty())
        run_adjoint(vec_sol);

      info.close();
      return 0;
    }

    // FP64 MG-PCG / MG-Richardson exactly as composed in applications/poisson_dirichlet.cpp:152-190
    template<typename Solver_>
    void configure(Solver_& s) const
    {
      s.set_tol_rel(cfg.tol);
      s.set_max_iter(Index(cfg.maxit));
      if(!cfg.quiet) s.set_plot_mode(Solver::PlotMode::iter);
    }

    // MultiGrid with the configured cycle and coarse-grid correction (multigrid.hpp:1066, 1089-1104)
    template<typename H_>
    auto make_multigrid(std::shared_ptr<H_> hier) const
      -> decltype(Solver::new_multigrid(hier, Solver::MultiGridCycle::V))
    {
      Solver::MultiGridCycle cyc = Solver::MultiGridCycle::V;
      if(cfg.cycle == "f") cyc = Solver::MultiGridCycle::F;
      else if(cfg.cycle == "w") cyc = Solver::MultiGridCycle::W;
      auto mg = Solver::new_multigrid(hier, cyc);
      if(cfg.cgc == "energy") mg->set_adapt_cgc(Solver::MultiGridAdaptCGC::MinEnergy);
      else if(cfg.cgc == "defect") mg->set_adapt_cgc(Solver::MultiGridAdaptCGC::MinDefect);
      return mg;
    }

    template<typename M_, typename F_, typename T_, typename LvlGet_>
    std::shared_ptr<Solver::MultiGridHierarchy<M_, F_, T_>> build_hierarchy(LvlGet_ get) const
    {
      auto hier = std::make_shared<Solver::MultiGridHierarchy<M_, F_, T_>>(levels.size());
      for(std::size_t i(0); i < levels.size(); ++i)
      {
        const M_& a = std::get<0>(get(*levels.at(i)));
        const F_& f = std::get<1>(get(*levels.at(i)));
        const T_& t = std::get<2>(get(*levels.at(i)));
        auto jac = Solver::new_jacobi_precond(a, f, typename M_::DataType(cfg.omega_jac));
        auto smoother = Solver::new_richardson(a, f, typename M_::DataType(cfg.omega_rich), jac);
        smoother->set_min_iter(Index(cfg.nu));
        smoother->set_max_iter(Index(cfg.nu));
        if(i + 1 < levels.size())
          hier->push_level(a, f, t, smoother, smoother, smoother);
        else
        {
          if(cfg.coarse == "direct")
            hier->push_level(a, f, std::make_shared<DenseDirectSolver<M_, F_>>(a, f));
          else if(cfg.coarse == "pcg")
            hier->push_level(a, f, Solver::new_pcg(a, f));
          else if(cfg.coarse == "smoother")
            hier->push_level(a, f, smoother);
          else
            hier->push_level(a, f, std::shared_ptr<Solver::SolverBase<typename M_::VectorTypeL>>());
        }
      }
      return hier;
    }

    // Solver::solve from a zero initial guess, `warmup` times with one iteration (untimed), then
    // timed (TimeStamp around Solver::solve only, applications/poisson_dirichlet.cpp:198-208)
    // `repeat` times or until the budget would be exceeded; t = the last timed solve
    template<typename S_, typename M_, typename F_>
    void timed_solves(S_& solver, VectorType& vec_sol, const VectorType& vec_rhs, const M_& mat, const F_& filt,
                      std::vector<double>& hist, int& iters, int& status, double& t)
    {
      for(int w(0); w < cfg.warmup; ++w)
      {
        solver.set_max_iter(Index(1));
        vec_sol.format();
        Solver::solve(solver, vec_sol, vec_rhs, mat, filt);
      }
      solver.set_max_iter(Index(cfg.maxit));
      double total = 0.0;
      for(int r(0); r < std::max(1, cfg.repeat); ++r)
      {
        if(r > 0 && cfg.budget_s > 0.0 && total + t > cfg.budget_s)
          break;
        vec_sol.format();
        TimeStamp at;
        auto st = Solver::solve(solver, vec_sol, vec_rhs, mat, filt);
        t = at.elapsed_now();
        total += t;
        solve_times.push_back(t);
        hist = solver.hist; iters = int(solver.get_num_iter()); status = int(st);
      }
    }

    void solve_f64(VectorType& vec_sol, const VectorType& vec_rhs, std::vector<double>& hist, int& iters, int& status, double& t)
    {
      Level& top = *levels.front();
      auto hier = build_hierarchy<MatrixType, FilterType, TransferType>(
        [](Level& l) { return std::tie(l.matrix, l.filter, l.transfer); });
      auto mgv = make_multigrid(hier);
      hier->init();
      if(cfg.solver == "pcg")
      {
        auto solver = std::make_shared<RecPCG<MatrixType, FilterType>>(top.matrix, top.filter, mgv);
        configure(*solver);
        solver->init();
        timed_solves(*solver, vec_sol, vec_rhs, top.matrix, top.filter, hist, iters, status, t);
        solver->done();
      }
      else
      {
        auto solver = std::make_shared<RecRichardson<MatrixType, FilterType>>(top.matrix, top.filter, cfg.omega_outer, mgv);
        configure(*solver);
        solver->init();
        timed_solves(*solver, vec_sol, vec_rhs, top.matrix, top.filter, hist, iters, status, t);
        solver->done();
      }
      hier->done();
    }

    // mixed precision: FP64 outer solver, ConvertPrecond (kernel/solver/convert_precond.hpp:41-120)
    // around an FP32 multigrid; "f16" additionally quantises every inner matrix to FP16 with a
    // per-level scale and dequantises it back into the FP32 containers.
    void solve_mixed(VectorType& vec_sol, const VectorType& vec_rhs, std::vector<double>& hist, int& iters, int& status, double& t)
    {
      for(auto& lp : levels)
      {
        Level& lv = *lp;
        lv.matrix_f.convert(lv.matrix);
        lv.filter_f.convert(lv.filter);
        lv.transfer_f.convert(lv.transfer);
        if(cfg.inner == "f16")
        {
          const double* v64 = lv.matrix.val();
          float* v32 = lv.matrix_f.val();
          const Index nnz = lv.matrix.used_elements();
          double amax = 0.0;
          for(Index i(0); i < nnz; ++i) amax = std::max(amax, std::fabs(v64[i]));
          const double scale = (amax > 0.0) ? amax / 16384.0 : 1.0;
          const double inv = 1.0 / scale;
          for(Index i(0); i < nnz; ++i)
          {
            _Float16 h = (_Float16)(v64[i] * inv);
            v32[i] = float(h) * float(scale);
          }
        }
      }
      Level& top = *levels.front();
      auto hier = build_hierarchy<MatrixTypeF, FilterTypeF, TransferTypeF>(
        [](Level& l) { return std::tie(l.matrix_f, l.filter_f, l.transfer_f); });
      auto mgv = make_multigrid(hier);
      auto conv = Solver::new_convert_precond<VectorType, VectorTypeF>(mgv);
      hier->init();
      if(cfg.solver == "pcg")
      {
        auto solver = std::make_shared<RecPCG<MatrixType, FilterType>>(top.matrix, top.filter, conv);
        configure(*solver);
        solver->init();
        timed_solves(*solver, vec_sol, vec_rhs, top.matrix, top.filter, hist, iters, status, t);
        solver->done();
      }
      else
      {
        auto solver = std::make_shared<RecRichardson<MatrixType, FilterType>>(top.matrix, top.filter, cfg.omega_outer, conv);
        configure(*solver);
        solver->init();
        timed_solves(*solver, vec_sol, vec_rhs, top.matrix, top.filter, hist, iters, status, t);
        solver->done();
      }
      hier->done();
    }

    // adjoint: A lambda = filter(u - u_target); dJ/dk_e = -int_e grad(lambda) . grad(u)
    void run_adjoint(const VectorType& vec_u)
    {
      Level& top = *levels.front();
      const Index N = Index(1) << top.lvl;
      const auto lat = dof_lattice(top, N);
      const auto tgt = read_f64(cfg.target);
      const Index n = top.space.get_num_dofs();
      VectorType vec_g(n), vec_lam(n);
      double J = 0.0;
      for(Index i(0); i < n; ++i)
      {
        const double d = vec_u(i) - tgt.at(lat[i]);
        vec_g(i, d);
        J += 0.5 * d * d;
      }
      top.filter.filter_def(vec_g);
      vec_lam.format();
      std::vector<double> hist; int iters = 0, status = 0; double t = 0.0;
      Config sub = cfg;
      solve_f64(vec_lam, vec_g, hist, iters, status, t);
      write_f64(cfg.out + ".lambda", std::vector<double>(vec_lam.elements(), vec_lam.elements() + n));

      // element gradient with the reference's own evaluators (same loop structure as
      // kernel/assembly/error_computer.hpp:467-520)
      typedef Assembly::AsmTraits1<double, SpaceType, TrafoTags::none, SpaceTags::grad> AsmTraits;
      Cubature::DynamicFactory cubature("auto-degree:5");
      typename AsmTraits::CubatureRuleType cubature_rule(Cubature::ctor_factory, cubature);
      const typename AsmTraits::TrafoType& trafo = top.space.get_trafo();
      typename AsmTraits::TrafoEvaluator trafo_eval(trafo);
      typename AsmTraits::SpaceEvaluator space_eval(top.space);
      typename AsmTraits::DofMapping dof_mapping(top.space);
      typename AsmTraits::TrafoEvalData trafo_data;
      typename AsmTraits::SpaceEvalData space_data;
      typename AsmTraits::LocalVectorType lu, ll;
      typename VectorType::GatherAxpy gu(vec_u), gl(vec_lam);
      Index ne = 1; for(int d(0); d < dim; ++d) ne *= N;
      std::vector<double> grad(ne, 0.0);
      for(typename AsmTraits::CellIterator cell(trafo_eval.begin()); cell != trafo_eval.end(); ++cell)
      {
        lu.format(); ll.format();
        dof_mapping.prepare(cell);
        gu(lu, dof_mapping);
        gl(ll, dof_mapping);
        dof_mapping.finish();
        trafo_eval.prepare(cell);
        space_eval.prepare(trafo_eval);
        const int nld = space_eval.get_num_local_dofs();
        double acc = 0.0;
        for(int k(0); k < cubature_rule.get_num_points(); ++k)
        {
          trafo_eval(trafo_data, cubature_rule.get_point(k));
          space_eval(space_data, trafo_data);
          double gu_[3] = {0,0,0}, gl_[3] = {0,0,0};
          for(int i(0); i < nld; ++i)
            for(int d(0); d < dim; ++d)
            {
              gu_[d] += lu[i] * space_data.phi[i].grad[d];
              gl_[d] += ll[i] * space_data.phi[i].grad[d];
            }
          double dd = 0.0;
          for(int d(0); d < dim; ++d) dd += gu_[d] * gl_[d];
          acc += trafo_data.jac_det * cubature_rule.get_weight(k) * dd;
        }
        space_eval.finish();
        trafo_eval.finish();
        grad[cell_lex(top.mesh, Index(cell), N)] = -acc;
      }
      write_f64(cfg.out + ".grad", grad);
      info << "J " << J << "\n";
      info << "adj_iters " << iters << "\n";
    }
  };
} // namespace RefDriver

int main(int argc, char** argv)
{
  Runtime::initialise(argc, argv);
  RefDriver::Config cfg;
  for(int i = 1; i < argc; ++i)
  {
    std::string a = argv[i];
    auto next = [&]() -> std::string { if(i + 1 >= argc) { std::cerr << "missing value for " << a << std::endl; std::exit(2); } return argv[++i]; };
    if(a == "--dim") cfg.dim = std::atoi(next().c_str());
    else if(a == "--degree") cfg.degree = std::atoi(next().c_str());
    else if(a == "--level") cfg.level = std::atoi(next().c_str());
    else if(a == "--level-min") cfg.level_min = std::atoi(next().c_str());
    else if(a == "--rhs") cfg.rhs = next();
    else if(a == "--kfile") cfg.kfile = next();
    else if(a == "--solver") cfg.solver = next();
    else if(a == "--nu") cfg.nu = std::atoi(next().c_str());
    else if(a == "--omega-jac") cfg.omega_jac = std::atof(next().c_str());
    else if(a == "--omega-rich") cfg.omega_rich = std::atof(next().c_str());
    else if(a == "--omega-outer") cfg.omega_outer = std::atof(next().c_str());
    else if(a == "--coarse") cfg.coarse = next();
    else if(a == "--tol") cfg.tol = std::atof(next().c_str());
    else if(a == "--maxit") cfg.maxit = std::atoi(next().c_str());
    else if(a == "--inner") cfg.inner = next();
    else if(a == "--cycle") cfg.cycle = next();
    else if(a == "--cgc") cfg.cgc = next();
    else if(a == "--target") cfg.target = next();
    else if(a == "--out") cfg.out = next();
    else if(a == "--dump-matrices") cfg.dump_matrices = true;
    else if(a == "--feat-files") cfg.dump_matrices = cfg.feat_files = true;
    else if(a == "--quiet") cfg.quiet = true;
    else if(a == "--repeat") cfg.repeat = std::atoi(next().c_str());
    else if(a == "--budget-s") cfg.budget_s = std::atof(next().c_str());
    else if(a == "--warmup") cfg.warmup = std::atoi(next().c_str());
    else { std::cerr << "unknown option " << a << std::endl; return 2; }
  }
  int rc = 0;
  if(cfg.dim == 2 && cfg.degree == 1)
    rc = RefDriver::Runner<Shape::Hypercube<2>, Space::Lagrange1::Element>(cfg).run();
  else if(cfg.dim == 2 && cfg.degree == 2)
    rc = RefDriver::Runner<Shape::Hypercube<2>, Space::Lagrange2::Element>(cfg).run();
  else if(cfg.dim == 3 && cfg.degree == 1)
    rc = RefDriver::Runner<Shape::Hypercube<3>, Space::Lagrange1::Element>(cfg).run();
  else if(cfg.dim == 3 && cfg.degree == 2)
    rc = RefDriver::Runner<Shape::Hypercube<3>, Space::Lagrange2::Element>(cfg).run();
  else { std::cerr << "unsupported dim/degree" << std::endl; rc = 2; }
  Runtime::finalise();
  return rc;
}
