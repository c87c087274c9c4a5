// Runs the reference's own LAFEM arch declarations for Mem::CUDA, bound onto libfeat3_b200 by
// feat3_b200/shim/feat_arch_cuda.cpp, on cudaMalloc'd buffers and compares every result with
// the reference's own Mem::Main templates (kernel/lafem/arch/*_generic.hpp) on the same inputs.
// Built against the reference headers by oracle/Makefile (target `shim`); run by
// tests/test_feat_shim.py on a GPU. Prints one line per check and exits 0 when all pass.
#include <kernel/lafem/arch/apply.hpp>
#include <kernel/lafem/arch/axpy.hpp>
#include <kernel/lafem/arch/component_invert.hpp>
#include <kernel/lafem/arch/component_product.hpp>
#include <kernel/lafem/arch/diagonal.hpp>
#include <kernel/lafem/arch/dot_product.hpp>
#include <kernel/lafem/arch/norm.hpp>
#include <kernel/lafem/arch/scale.hpp>
#include <kernel/lafem/arch/unit_filter.hpp>
#include <kernel/util/exception.hpp>

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <random>
#include <string>
#include <vector>

using namespace FEAT;
using namespace FEAT::LAFEM::Arch;
using FEAT::Index;

namespace
{
  int failures = 0;

  void check(const std::string& name, double err, double tol)
  {
    const bool ok = std::isfinite(err) && err <= tol;
    std::printf("%s %s err %.3e tol %.1e\n", ok ? "ok" : "FAIL", name.c_str(), err, tol);
    if(!ok) ++failures;
  }

  template<typename T>
  double relerr(const std::vector<T>& a, const std::vector<T>& b)
  {
    double num = 0.0, den = 0.0;
    for(std::size_t i(0); i < a.size(); ++i)
    {
      const double d = double(a[i]) - double(b[i]);
      num += d * d;
      den += double(b[i]) * double(b[i]);
    }
    return std::sqrt(num / std::max(den, 1e-300));
  }

  void cuda_ok(cudaError_t e, const char* what)
  {
    if(e != cudaSuccess)
    {
      std::printf("FAIL cuda %s: %s\n", what, cudaGetErrorString(e));
      std::exit(2);
    }
  }

  template<typename T>
  struct Dev
  {
    T* p = nullptr;
    std::size_t n = 0;
    explicit Dev(const std::vector<T>& h) : n(h.size())
    {
      cuda_ok(cudaMalloc((void**)&p, std::max<std::size_t>(n, 1) * sizeof(T)), "malloc");
      if(n) cuda_ok(cudaMemcpy(p, h.data(), n * sizeof(T), cudaMemcpyHostToDevice), "upload");
    }
    ~Dev() { cudaFree(p); }
    std::vector<T> get() const
    {
      std::vector<T> h(n);
      cuda_ok(cudaDeviceSynchronize(), "sync");
      if(n) cuda_ok(cudaMemcpy(h.data(), p, n * sizeof(T), cudaMemcpyDeviceToHost), "download");
      return h;
    }
  };

  // a random sparse matrix: every row has its diagonal and 2..14 further entries, some rows
  // empty (stored as no entries), columns sorted within a row
  template<typename IT_>
  void make_csr(Index rows, Index cols, std::vector<IT_>& rp, std::vector<IT_>& ci, std::vector<double>& va,
                std::mt19937_64& rng)
  {
    std::uniform_int_distribution<Index> len(2, 14), col(0, cols - 1);
    std::uniform_real_distribution<double> val(-1.0, 1.0);
    rp.assign(1, 0);
    for(Index r(0); r < rows; ++r)
    {
      std::vector<Index> c;
      if(r % 97 != 13)
      {
        c.push_back(r < cols ? r : col(rng));
        for(Index k(0), m(len(rng)); k < m; ++k) c.push_back(col(rng));
      }
      std::sort(c.begin(), c.end());
      c.erase(std::unique(c.begin(), c.end()), c.end());
      for(Index x : c) { ci.push_back(IT_(x)); va.push_back(val(rng)); }
      rp.push_back(IT_(ci.size()));
    }
  }

  // FEAT's SELL-C layout (kernel/lafem/sparse_matrix_ell.hpp:38-63): chunk c holds rows
  // c*C..c*C+C-1, entry j of row c*C+l at cs[c] + j*C + l, chunk length cl[c] = its longest row
  template<typename IT_>
  void to_ell(const std::vector<IT_>& rp, const std::vector<IT_>& ci, const std::vector<double>& va, Index C,
              std::vector<IT_>& cs, std::vector<IT_>& cl, std::vector<IT_>& ec, std::vector<double>& ev)
  {
    const Index rows = rp.size() - 1, nch = (rows + C - 1) / C;
    cs.assign(nch + 1, 0);
    cl.assign(nch, 0);
    for(Index c(0); c < nch; ++c)
    {
      Index m = 0;
      for(Index l(0); l < C && c * C + l < rows; ++l) m = std::max<Index>(m, rp[c * C + l + 1] - rp[c * C + l]);
      cl[c] = IT_(m);
      cs[c + 1] = IT_(cs[c] + m * C);
    }
    ec.assign(cs[nch], 0);
    ev.assign(cs[nch], 0.0);
    for(Index r(0); r < rows; ++r)
    {
      const Index c = r / C, l = r % C;
      for(Index j(0); j < Index(rp[r + 1] - rp[r]); ++j)
      {
        ec[cs[c] + j * C + l] = ci[rp[r] + j];
        ev[cs[c] + j * C + l] = va[rp[r] + j];
      }
    }
  }

  template<typename DT_, typename IT_>
  void run_csr(const char* tag, Index rows, Index cols, std::mt19937_64& rng, double tol)
  {
    std::vector<IT_> rp, ci;
    std::vector<double> va64;
    make_csr(rows, cols, rp, ci, va64, rng);
    std::vector<DT_> va(va64.begin(), va64.end());
    std::uniform_real_distribution<double> u(-1.0, 1.0);
    std::vector<DT_> x(cols), y(rows), xt(rows), yt(cols);
    for(auto& v : x) v = DT_(u(rng));
    for(auto& v : y) v = DT_(u(rng));
    for(auto& v : xt) v = DT_(u(rng));
    for(auto& v : yt) v = DT_(u(rng));
    Dev<DT_> dval(va), dx(x), dy(y), dxt(xt), dyt(yt);
    Dev<IT_> dci(ci), drp(rp);
    const Index nnz = ci.size();
    const DT_ alphas[3] = {DT_(0), DT_(-1), DT_(0.37)};
    for(DT_ a : alphas)
    {
      for(DT_ b : {DT_(1), DT_(0), DT_(-0.5)})
      {
        // r = b*y + a*A*x (Apply<Mem::Main>::csr_generic, apply_generic.hpp:25-70)
        std::vector<DT_> ref(rows);
        Apply<Mem::Main>::csr_generic(ref.data(), a, x.data(), b, y.data(), va.data(), ci.data(), rp.data(), rows, cols,
                                      nnz, false);
        Dev<DT_> dr{std::vector<DT_>(rows, DT_(7))};
        Apply<Mem::CUDA>::csr(dr.p, a, dx.p, b, dy.p, dval.p, dci.p, drp.p, rows, cols, nnz, false);
        check(std::string(tag) + " csr a=" + std::to_string(double(a)) + " b=" + std::to_string(double(b)),
              relerr(dr.get(), ref), tol);
        // transposed: r (cols) = b*y + a*A^T*x
        std::vector<DT_> reft(cols);
        if(a != DT_(0))
        {
          Apply<Mem::Main>::csr_generic(reft.data(), a, xt.data(), b, yt.data(), va.data(), ci.data(), rp.data(), rows,
                                        cols, nnz, true);
          Dev<DT_> drt{std::vector<DT_>(cols, DT_(7))};
          Apply<Mem::CUDA>::csr(drt.p, a, dxt.p, b, dyt.p, dval.p, dci.p, drp.p, rows, cols, nnz, true);
          check(std::string(tag) + " csr^T a=" + std::to_string(double(a)) + " b=" + std::to_string(double(b)),
                relerr(drt.get(), reft), 10 * tol);
        }
      }
    }
    // r aliasing y (the containers' apply(r, x, r, alpha) form)
    {
      std::vector<DT_> ref(y);
      Apply<Mem::Main>::csr_generic(ref.data(), DT_(-1), x.data(), DT_(1), ref.data(), va.data(), ci.data(), rp.data(),
                                    rows, cols, nnz, false);
      Dev<DT_> dr(y);
      Apply<Mem::CUDA>::csr(dr.p, DT_(-1), dx.p, DT_(1), dr.p, dval.p, dci.p, drp.p, rows, cols, nnz, false);
      check(std::string(tag) + " csr r==y", relerr(dr.get(), ref), tol);
    }
    // FEAT's SELL-C (ELL) form of the same square part, C = 32 (sparse_matrix_ell.hpp:387)
    if(rows == cols)
    {
      std::vector<IT_> cs, cl, ec;
      std::vector<double> ev64;
      to_ell(rp, ci, va64, 32, cs, cl, ec, ev64);
      std::vector<DT_> ev(ev64.begin(), ev64.end());
      std::vector<DT_> ref(rows);
      Apply<Mem::Main>::ell_generic(ref.data(), DT_(0.37), x.data(), DT_(-0.5), y.data(), ev.data(), ec.data(),
                                    cs.data(), cl.data(), 32, rows);
      Dev<DT_> dev{ev}, dr{std::vector<DT_>(rows, DT_(7))};
      Dev<IT_> dec(ec), dcs(cs), dcl(cl);
      Apply<Mem::CUDA>::ell(dr.p, DT_(0.37), dx.p, DT_(-0.5), dy.p, dev.p, dec.p, dcs.p, dcl.p, 32, rows);
      check(std::string(tag) + " ell", relerr(dr.get(), ref), tol);
      // diagonals (Diagonal<Mem::Main>::csr_generic / ell_generic)
      std::vector<DT_> dref(rows), dref_e(rows);
      Diagonal<Mem::Main>::csr_generic(dref.data(), va.data(), ci.data(), rp.data(), rows);
      Diagonal<Mem::Main>::ell_generic(dref_e.data(), ev.data(), ec.data(), cs.data(), cl.data(), 32, rows);
      Dev<DT_> dd{std::vector<DT_>(rows, DT_(7))}, dde{std::vector<DT_>(rows, DT_(7))};
      Diagonal<Mem::CUDA>::csr(dd.p, dval.p, dci.p, drp.p, rows);
      Diagonal<Mem::CUDA>::ell(dde.p, dev.p, dec.p, dcs.p, dcl.p, 32, rows);
      check(std::string(tag) + " diagonal csr", relerr(dd.get(), dref), 0.0);
      check(std::string(tag) + " diagonal ell", relerr(dde.get(), dref_e), 0.0);
    }
  }

  template<typename DT_, typename IT_>
  void run_filter(const char* tag, Index n, std::mt19937_64& rng)
  {
    std::vector<IT_> idx;
    std::vector<DT_> sv, v(n);
    std::uniform_real_distribution<double> u(-1.0, 1.0);
    for(Index i(0); i < n; i += 3) { idx.push_back(IT_(i)); sv.push_back(DT_(u(rng))); }
    for(auto& a : v) a = DT_(u(rng));
    std::vector<DT_> rhs(v), def(v);
    UnitFilter<Mem::Main>::filter_rhs_generic(rhs.data(), sv.data(), idx.data(), idx.size());
    UnitFilter<Mem::Main>::filter_def_generic(def.data(), idx.data(), idx.size());
    Dev<DT_> dv1(v), dv2(v), dsv(sv);
    Dev<IT_> didx(idx);
    UnitFilter<Mem::CUDA>::filter_rhs(dv1.p, dsv.p, didx.p, idx.size());
    UnitFilter<Mem::CUDA>::filter_def(dv2.p, didx.p, idx.size());
    check(std::string(tag) + " unit filter rhs", relerr(dv1.get(), rhs), 0.0);
    check(std::string(tag) + " unit filter def", relerr(dv2.get(), def), 0.0);
  }

  template<typename DT_>
  void run_blas1(const char* tag, Index n, std::mt19937_64& rng, double tol)
  {
    std::uniform_real_distribution<double> u(0.5, 1.5);
    std::vector<DT_> x(n), y(n);
    for(auto& v : x) v = DT_(u(rng));
    for(auto& v : y) v = DT_(u(rng));
    Dev<DT_> dx(x), dy(y);
    // reductions: the reference's template on the same values held exactly in FP64 (its FP32
    // instance sums a million terms sequentially in FP32, ~1e-5 off; the library sums in FP64)
    const std::vector<double> x64(x.begin(), x.end()), y64(y.begin(), y.end());
    const double dref = DotProduct<Mem::Main>::value_generic(x64.data(), y64.data(), n);
    const DT_ dgpu = DotProduct<Mem::CUDA>::value(dx.p, dy.p, n);
    check(std::string(tag) + " dot", std::abs(double(dgpu) - dref) / std::abs(dref), tol);
    const double nref = Norm2<Mem::Main>::value_generic(x64.data(), n);
    const DT_ ngpu = Norm2<Mem::CUDA>::value(dx.p, n);
    check(std::string(tag) + " norm2", std::abs(double(ngpu) - nref) / nref, tol);
    std::vector<DT_> r1(n), r2(n), r3(n), r4(n);
    Axpy<Mem::Main>::dv_generic(r1.data(), DT_(-0.75), x.data(), y.data(), n);
    ComponentProduct<Mem::Main>::value_generic(r2.data(), x.data(), y.data(), n);
    ComponentInvert<Mem::Main>::value_generic(r3.data(), x.data(), DT_(0.5), n);
    Scale<Mem::Main>::value_generic(r4.data(), x.data(), DT_(3.25), n);
    const std::vector<DT_> zero(n, DT_(0));
    Dev<DT_> g1{zero}, g2{zero}, g3{zero}, g4{zero};
    Axpy<Mem::CUDA>::dv(g1.p, DT_(-0.75), dx.p, dy.p, n);
    ComponentProduct<Mem::CUDA>::value(g2.p, dx.p, dy.p, n);
    ComponentInvert<Mem::CUDA>::value(g3.p, dx.p, DT_(0.5), n);
    Scale<Mem::CUDA>::value(g4.p, dx.p, DT_(3.25), n);
    check(std::string(tag) + " axpy", relerr(g1.get(), r1), tol);
    check(std::string(tag) + " component_product", relerr(g2.get(), r2), tol);
    check(std::string(tag) + " component_invert", relerr(g3.get(), r3), tol);
    check(std::string(tag) + " scale", relerr(g4.get(), r4), tol);
  }
} // namespace

int main()
{
  std::mt19937_64 rng(20261203);
  run_csr<double, unsigned int>("f64/u32", 40000, 40000, rng, 1e-13);
  run_csr<double, unsigned long>("f64/u64", 40000, 40000, rng, 1e-13);
  run_csr<double, unsigned long>("f64/u64 rect", 30000, 41000, rng, 1e-13);
  run_csr<float, unsigned int>("f32/u32", 40000, 40000, rng, 1e-5);
  run_csr<float, unsigned long>("f32/u64", 40000, 40000, rng, 1e-5);
  run_filter<double, unsigned int>("f64/u32", 50000, rng);
  run_filter<double, unsigned long>("f64/u64", 50000, rng);
  run_filter<float, unsigned long>("f32/u64", 50000, rng);
  run_blas1<double>("f64", 1000003, rng, 1e-13);
  run_blas1<float>("f32", 1000003, rng, 1e-6);
  // a failing call reaches the caller as the reference's InternalError
  bool thrown = false;
  try
  {
    Apply<Mem::CUDA>::csr<double>(nullptr, 1.0, nullptr, 1.0, nullptr, nullptr, (const unsigned long*)nullptr,
                                  (const unsigned long*)nullptr, 10, 10, 10, false);
  }
  catch(const InternalError&)
  {
    thrown = true;
  }
  check("invalid arguments -> InternalError", thrown ? 0.0 : 1.0, 0.0);
  std::printf("%s: %d failure(s)\n", failures ? "FAILED" : "PASSED", failures);
  return failures ? 1 : 0;
}
