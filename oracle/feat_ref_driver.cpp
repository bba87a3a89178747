// Oracle driver over the reference's own public API (TEST INFRASTRUCTURE ONLY).
//
// This program is compiled by oracle/Makefile against the FEAT3 sources (headers plus the few
// runtime .cpp files) and linked into oracle/_ref/feat_oracle.  It is the reference side of the
// parity tests and the CPU baseline of bench.py: it builds the Poisson multigrid problems with
// FEAT's own mesh refinement, Q1 assembly and grid transfer, solves them with FEAT's own
// Solver::PCG + Solver::MultiGrid + Solver::Richardson + Solver::JacobiPrecond, and dumps the
// matrices, vectors and iterates as .npy files.  Nothing in the product links or runs it.
//
// The setup follows the reference's tutorial (tutorials/tutorial_05_multigrid.cpp:211-312 for
// mesh, assembly and transfer; :363-460 for the hierarchy and solver), with PCG as the outer solver
// (kernel/solver/pcg.hpp:188-286), Richardson(omega=1)+Jacobi(omega) smoothers with
// min_iter = max_iter = steps (kernel/solver/richardson.hpp:160-228,
// kernel/solver/jacobi_precond.hpp:136-165) and an exact dense coarse solve (the class
// CoarseInverseSolver below; the reference offers no third-party-free direct solver).
//
// Usage:
// Built a second time with -DFEAT_HAVE_CUDA -DFEATB200_BACKEND and the library's FEAT binding
// (feat3.doxytest_b200/feat/featb200_backend.cpp in place of FEAT's CUDA backend, linked with
// libfeatb200.so) into oracle/_ref/feat_b200: the same program, where FEAT's containers hold managed
// memory and two more options exist:
//   --backend b200   FEAT's own PCG + MultiGrid with every LAFEM op dispatched to the CUDA backend
//                    (Backend::set_preferred_backend(PreferredBackend::cuda)), i.e. to the library
//   --b200-solver    the whole solve handed to the library's solver object (featb200_solver.hpp)
// And a third time with -DFEAT_HAVE_CUDA and FEAT's own CUDA backend (its kernel/util/cuda_util.cu and
// kernel/lafem/arch/*.cu compiled by nvcc, cuSPARSE / cuBLAS) into oracle/_ref/feat_cuda, where
//   --backend cuda   runs FEAT's own PCG + MultiGrid with every LAFEM op on FEAT's GPU kernels
// (the reference's GPU path, for a timing column beside the library).
//
//   feat_oracle fd M D DIR     (the reference's basic_solver-test problem, see run_fd)
//   feat_oracle solve --dim D --level L --out DIR [--rhs sine|gauss] [--params FILE]
//                     [--kappa FILE] [--omega W] [--steps S] [--tol T] [--iterates K]
//                     [--vcycle] [--dump-levels] [--time REPS] [--no-dump] [--cycle v|f|w]
//                     [--cgc fixed|energy|defect] [--smoother jacobi|sor|ssor] [--sor-omega W]
//
// The params files are written by the caller (tests/bench) so that the reference and the GPU
// path consume exactly the same Gaussian and random-field coefficients.

#include <kernel/runtime.hpp>
#include <kernel/util/string.hpp>
#include <kernel/geometry/boundary_factory.hpp>
#include <kernel/geometry/conformal_mesh.hpp>
#include <kernel/geometry/common_factories.hpp>
#include <kernel/geometry/mesh_part.hpp>
#include <kernel/trafo/standard/mapping.hpp>
#include <kernel/space/lagrange1/element.hpp>
#include <kernel/cubature/dynamic_factory.hpp>
#include <kernel/analytic/common.hpp>
#include <kernel/analytic/lambda_function.hpp>
#include <kernel/assembly/symbolic_assembler.hpp>
#include <kernel/assembly/unit_filter_assembler.hpp>
#include <kernel/assembly/domain_assembler.hpp>
#include <kernel/assembly/domain_assembler_helpers.hpp>
#include <kernel/assembly/common_operators.hpp>
#include <kernel/assembly/common_functionals.hpp>
#include <kernel/assembly/grid_transfer.hpp>
#include <kernel/assembly/bilinear_operator.hpp>
#include <kernel/lafem/dense_vector.hpp>
#include <kernel/lafem/sparse_matrix_csr.hpp>
#include <kernel/lafem/unit_filter.hpp>
#include <kernel/lafem/transfer.hpp>
#include <kernel/lafem/pointstar_factory.hpp>
#include <kernel/lafem/none_filter.hpp>
#include <kernel/solver/pcg.hpp>
#include <kernel/solver/richardson.hpp>
#include <kernel/solver/jacobi_precond.hpp>
#include <kernel/solver/sor_precond.hpp>
#include <kernel/solver/ssor_precond.hpp>
#include <kernel/solver/multigrid.hpp>
#ifdef FEATB200_BACKEND
#include <kernel/backend.hpp>
#include <featb200_solver.hpp>
#endif

#include <algorithm>
#include <chrono>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstring>
#include <deque>
#include <fstream>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

using namespace FEAT;

namespace Oracle
{
  typedef double DataType;
  typedef Index IndexType;
  typedef LAFEM::DenseVector<DataType, IndexType> VectorType;
  typedef LAFEM::SparseMatrixCSR<DataType, IndexType> MatrixType;
  typedef LAFEM::UnitFilter<DataType, IndexType> FilterType;
  typedef LAFEM::Transfer<MatrixType> TransferType;

  // ---------------------------------------------------------------- .npy output
  static void write_npy(const std::string& path, const char* descr, std::size_t elem,
    const void* data, std::size_t count)
  {
    std::string header = std::string("{'descr': '") + descr + "', 'fortran_order': False, 'shape': (" +
      std::to_string(count) + ",), }";
    std::size_t total = 10 + header.size() + 1;
    std::size_t pad = (64 - total % 64) % 64;
    header.append(pad, ' ');
    header.push_back('\n');
    std::ofstream f(path, std::ios::binary);
    if(!f)
    {
      std::fprintf(stderr, "cannot write %s\n", path.c_str());
      std::exit(2);
    }
    const char magic[8] = {'\x93', 'N', 'U', 'M', 'P', 'Y', 1, 0};
    f.write(magic, 8);
    unsigned short hl = (unsigned short)header.size();
    f.write(reinterpret_cast<const char*>(&hl), 2);
    f.write(header.data(), std::streamsize(header.size()));
    f.write(reinterpret_cast<const char*>(data), std::streamsize(elem * count));
  }

  static void dump_vec(const std::string& path, const VectorType& v)
  {
    write_npy(path, "<f8", 8, v.elements(), v.size());
  }

  static void dump_csr(const std::string& prefix, const MatrixType& a)
  {
    std::vector<unsigned long long> rp(a.row_ptr(), a.row_ptr() + a.rows() + 1);
    std::vector<unsigned long long> ci(a.col_ind(), a.col_ind() + a.used_elements());
    write_npy(prefix + "_row_ptr.npy", "<u8", 8, rp.data(), rp.size());
    write_npy(prefix + "_col_ind.npy", "<u8", 8, ci.data(), ci.size());
    write_npy(prefix + "_val.npy", "<f8", 8, a.val(), a.used_elements());
    unsigned long long shape[2] = {a.rows(), a.columns()};
    write_npy(prefix + "_shape.npy", "<u8", 8, shape, 2);
  }

  // ---------------------------------------------------------------- problem coefficients
  // Gaussian sum f(x) = sum_k a_k exp(-|x-c_k|^2 / (2 w_k^2)); one line per Gaussian:
  //   c_1 .. c_dim  w  a
  struct GaussParams
  {
    int dim = 2;
    std::vector<std::vector<double>> rows;
  };

  static GaussParams read_gauss(const std::string& file, int dim)
  {
    GaussParams p;
    p.dim = dim;
    std::ifstream f(file);
    std::string line;
    while(std::getline(f, line))
    {
      if(line.empty() || line[0] == '#')
        continue;
      std::istringstream is(line);
      std::vector<double> r;
      double v;
      while(is >> v)
        r.push_back(v);
      if(int(r.size()) == dim + 2)
        p.rows.push_back(r);
    }
    return p;
  }

  // Random field g(x,y) = s * sum_{i,j} (xi_ij cos t + eta_ij sin t) / (kx_i^2 + ky_j^2),
  // t = 2 pi (kx_i x + ky_j y); kappa = exp(g).  File: first line "K s", then K lines with
  // kx_i, then K lines with ky_j, then K*K lines "xi eta" (row-major in i, then j).
  struct FieldParams
  {
    int k = 0;
    double s = 0.0;
    std::vector<double> kx, ky, xi, eta;
    bool active() const { return k > 0; }

    double g(double x, double y) const
    {
      // separable evaluation: for each i, h_i = sum_j c_ij e^{2 pi i ky_j y}; g = s * sum_i Re(h_i e^{2 pi i kx_i x})
      const double tp = 2.0 * M_PI;
      double acc = 0.0;
      for(int i = 0; i < k; ++i)
      {
        double hr = 0.0, hi = 0.0;
        for(int j = 0; j < k; ++j)
        {
          const double den = kx[i] * kx[i] + ky[j] * ky[j];
          if(den == 0.0)
            continue;
          const double cy = std::cos(tp * ky[j] * y), sy = std::sin(tp * ky[j] * y);
          const double a = xi[std::size_t(i * k + j)] / den, b = eta[std::size_t(i * k + j)] / den;
          // (a - i b) (cy + i sy)
          hr += a * cy + b * sy;
          hi += a * sy - b * cy;
        }
        const double cx = std::cos(tp * kx[i] * x), sx = std::sin(tp * kx[i] * x);
        acc += hr * cx - hi * sx;
      }
      return s * acc;
    }
  };

  static FieldParams read_field(const std::string& file)
  {
    FieldParams p;
    std::ifstream f(file);
    if(!(f >> p.k >> p.s))
    {
      std::fprintf(stderr, "bad field file %s\n", file.c_str());
      std::exit(2);
    }
    p.kx.resize(std::size_t(p.k));
    p.ky.resize(std::size_t(p.k));
    for(auto& v : p.kx) f >> v;
    for(auto& v : p.ky) f >> v;
    p.xi.resize(std::size_t(p.k * p.k));
    p.eta.resize(std::size_t(p.k * p.k));
    for(std::size_t i = 0; i < p.xi.size(); ++i)
      f >> p.xi[i] >> p.eta[i];
    return p;
  }

  // -div(kappa grad u) operator: the Laplace bilinear form weighted by kappa at the cubature point,
  // written as a custom Assembly::BilinearOperator in the pattern of
  // tutorials/tutorial_03_andicore.cpp:131-260.
  class KappaLaplaceOperator :
    public Assembly::BilinearOperator
  {
  public:
    const FieldParams& field;
    explicit KappaLaplaceOperator(const FieldParams& f) : field(f) {}

    static constexpr TrafoTags trafo_config = TrafoTags::img_point;
    static constexpr SpaceTags test_config = SpaceTags::grad;
    static constexpr SpaceTags trial_config = SpaceTags::grad;

    template<typename AsmTraits_>
    class Evaluator :
      public Assembly::BilinearOperator::Evaluator<AsmTraits_>
    {
    public:
      typedef typename AsmTraits_::TrafoData TrafoData;
      typedef typename AsmTraits_::TrialBasisData TrialBasisData;
      typedef typename AsmTraits_::TestBasisData TestBasisData;
      typedef typename AsmTraits_::DataType DT;
      typedef DT ValueType;
    protected:
      const FieldParams& _field;
      DT _kappa;
    public:
      explicit Evaluator(const KappaLaplaceOperator& op) : _field(op.field), _kappa(1) {}
      void set_point(const TrafoData& tau)
      {
        _kappa = std::exp(_field.g(double(tau.img_point[0]), double(tau.img_point[1])));
      }
      ValueType eval(const TrialBasisData& phi, const TestBasisData& psi) const
      {
        return _kappa * dot(phi.grad, psi.grad);
      }
    };
  };

  // Exact coarse-grid solve: the inverse of the matrix restricted to the free (non-Dirichlet)
  // DOFs, formed once by Gauss-Jordan elimination with partial pivoting and applied as a dense
  // matrix-vector product in ascending column order.  Dirichlet entries of the output are zero.
  class CoarseInverseSolver :
    public Solver::SolverBase<VectorType>
  {
  public:
    const MatrixType& matrix;
    const FilterType& filter;
    std::vector<Index> free_dofs;
    std::vector<double> inv;

    CoarseInverseSolver(const MatrixType& a, const FilterType& f) : matrix(a), filter(f) {}
    virtual String name() const override { return "CoarseInverse"; }

    virtual void init_numeric() override
    {
      const Index n = matrix.rows();
      std::vector<char> dir(n, 0);
      const auto& fv = filter.get_filter_vector();
      for(Index k = 0; k < fv.used_elements(); ++k)
        dir[fv.indices()[k]] = 1;
      free_dofs.clear();
      for(Index i = 0; i < n; ++i)
        if(!dir[i]) free_dofs.push_back(i);
      const std::size_t m = free_dofs.size();
      std::vector<Index> pos(n, ~Index(0));
      for(std::size_t i = 0; i < m; ++i) pos[free_dofs[i]] = i;
      std::vector<double> a(m * m, 0.0);
      for(std::size_t i = 0; i < m; ++i)
      {
        const Index r = free_dofs[i];
        for(Index k = matrix.row_ptr()[r]; k < matrix.row_ptr()[r + 1]; ++k)
        {
          const Index c = matrix.col_ind()[k];
          if(pos[c] != ~Index(0)) a[i * m + pos[c]] = matrix.val()[k];
        }
      }
      inv.assign(m * m, 0.0);
      for(std::size_t i = 0; i < m; ++i) inv[i * m + i] = 1.0;
      for(std::size_t c = 0; c < m; ++c)
      {
        std::size_t p = c;
        for(std::size_t r = c + 1; r < m; ++r)
          if(std::fabs(a[r * m + c]) > std::fabs(a[p * m + c])) p = r;
        if(p != c)
          for(std::size_t j = 0; j < m; ++j)
          {
            std::swap(a[p * m + j], a[c * m + j]);
            std::swap(inv[p * m + j], inv[c * m + j]);
          }
        const double d = a[c * m + c];
        for(std::size_t j = 0; j < m; ++j)
        {
          a[c * m + j] /= d;
          inv[c * m + j] /= d;
        }
        for(std::size_t r = 0; r < m; ++r)
        {
          if(r == c) continue;
          const double f = a[r * m + c];
          if(f == 0.0) continue;
          for(std::size_t j = 0; j < m; ++j)
          {
            a[r * m + j] -= f * a[c * m + j];
            inv[r * m + j] -= f * inv[c * m + j];
          }
        }
      }
    }

    virtual Solver::Status apply(VectorType& vec_cor, const VectorType& vec_def) override
    {
      const std::size_t m = free_dofs.size();
      vec_cor.format();
      double* x = vec_cor.elements();
      const double* b = vec_def.elements();
      for(std::size_t i = 0; i < m; ++i)
      {
        double s = 0.0;
        for(std::size_t j = 0; j < m; ++j)
          s += inv[i * m + j] * b[free_dofs[j]];
        x[free_dofs[i]] = s;
      }
      return Solver::Status::success;
    }
  };

  struct Options
  {
    int dim = 2;
    std::string cycle = "v";   // multigrid cycle: v, f or w
    std::string cgc = "fixed"; // coarse-grid correction: fixed, energy or defect
    Index level = 7;
    Index level_min = 1;
    std::string out = ".";
    std::string rhs = "sine";
    std::string params;
    std::string kappa;
    double omega = 0.7;
    Index steps = 2;
    double tol = 1e-8;
    Index iterates = 0;
    bool vcycle = false;
    bool dump_levels = false;
    bool dump = true;
    int time_reps = 0;
    std::string smoother = "jacobi";   // the Richardson smoother's preconditioner: jacobi | sor | ssor
    double sor_omega = 1.0;            // SOR / SSOR damping
    std::string backend = "generic";   // generic | b200 (FEATB200_BACKEND builds) | cuda (CUDA builds)
    bool b200_solver = false;          // FEATB200_BACKEND builds only
  };

  template<int dim_>
  class Level
  {
  public:
    typedef Shape::Hypercube<dim_> ShapeType;
    typedef Geometry::ConformalMesh<ShapeType> MeshType;
    typedef Geometry::MeshPart<MeshType> MeshPartType;
    typedef Trafo::Standard::Mapping<MeshType> TrafoType;
    typedef Space::Lagrange1::Element<TrafoType> SpaceType;

    MeshType mesh;
    TrafoType trafo;
    SpaceType space;
    Assembly::DomainAssembler<TrafoType> domain_assembler;
    MatrixType matrix;
    FilterType filter;
    TransferType transfer;

    explicit Level(Geometry::Factory<MeshType>& factory) :
      mesh(factory), trafo(mesh), space(trafo), domain_assembler(trafo)
    {
    }
  };

  template<int dim_>
  int run(const Options& opt)
  {
    typedef Level<dim_> LevelType;
    typedef typename LevelType::MeshType MeshType;
    typedef typename LevelType::MeshPartType MeshPartType;

    const String cubature_name = "auto-degree:5";
    FieldParams field;
    if(!opt.kappa.empty())
    {
      if(dim_ != 2)
      {
        std::fprintf(stderr, "--kappa is implemented for 2D only\n");
        return 2;
      }
      field = read_field(opt.kappa);
    }

    auto t_setup = std::chrono::steady_clock::now();
    std::deque<std::shared_ptr<LevelType>> levels;
    {
      Geometry::RefinedUnitCubeFactory<MeshType> factory(opt.level_min);
      levels.push_front(std::make_shared<LevelType>(factory));
    }
    for(Index l = opt.level_min; l < opt.level; ++l)
    {
      Geometry::StandardRefinery<MeshType> factory(levels.front()->mesh);
      levels.push_front(std::make_shared<LevelType>(factory));
    }

    for(Index l = opt.level_min; l <= opt.level; ++l)
    {
      LevelType& lvl = *levels.at(std::size_t(opt.level - l));
      lvl.domain_assembler.compile_all_elements();
      Assembly::SymbolicAssembler::assemble_matrix_std1(lvl.matrix, lvl.space);
      lvl.matrix.format();
      if(field.active())
      {
        KappaLaplaceOperator op(field);
        Assembly::assemble_bilinear_operator_matrix_1(lvl.domain_assembler, lvl.matrix, op, lvl.space, cubature_name);
      }
      else
      {
        Assembly::Common::LaplaceOperator op;
        Assembly::assemble_bilinear_operator_matrix_1(lvl.domain_assembler, lvl.matrix, op, lvl.space, cubature_name);
      }
      Geometry::BoundaryFactory<MeshType> boundary_factory(lvl.mesh);
      MeshPartType boundary(boundary_factory);
      Assembly::UnitFilterAssembler<MeshType> unit_asm;
      unit_asm.add_mesh_part(boundary);
      unit_asm.assemble(lvl.filter, lvl.space);
    }
    for(Index l = opt.level_min; l < opt.level; ++l)
    {
      LevelType& fine = *levels.at(std::size_t(opt.level - l - 1));
      LevelType& coarse = *levels.at(std::size_t(opt.level - l));
      MatrixType& prol = fine.transfer.get_mat_prol();
      MatrixType& rest = fine.transfer.get_mat_rest();
      Assembly::SymbolicAssembler::assemble_matrix_2lvl(prol, fine.space, coarse.space);
      prol.format();
      Assembly::GridTransfer::assemble_prolongation_direct(prol, fine.space, coarse.space, cubature_name);
      rest = prol.transpose();
    }

    LevelType& top = *levels.front();
    VectorType vec_rhs = top.matrix.create_vector_r();
    vec_rhs.format();
    if(opt.rhs == "sine")
    {
      Analytic::Common::SineBubbleFunction<dim_> sol_function;
      Assembly::Common::LaplaceFunctional<decltype(sol_function)> force(sol_function);
      Assembly::assemble_linear_functional_vector(top.domain_assembler, vec_rhs, force, top.space, cubature_name);
    }
    else if(opt.rhs == "gauss")
    {
      GaussParams gp = read_gauss(opt.params, dim_);
      if(gp.rows.empty())
      {
        std::fprintf(stderr, "no Gaussians in %s\n", opt.params.c_str());
        return 2;
      }
      if constexpr(dim_ == 2)
      {
        auto f = Analytic::create_lambda_function_scalar_2d([&gp](double x, double y)
        {
          double s = 0.0;
          for(const auto& r : gp.rows)
          {
            const double dx = x - r[0], dy = y - r[1];
            s += r[3] * std::exp(-(dx * dx + dy * dy) / (2.0 * r[2] * r[2]));
          }
          return s;
        });
        Assembly::Common::ForceFunctional<decltype(f)> force(f);
        Assembly::assemble_linear_functional_vector(top.domain_assembler, vec_rhs, force, top.space, cubature_name);
      }
      else
      {
        auto f = Analytic::create_lambda_function_scalar_3d([&gp](double x, double y, double z)
        {
          double s = 0.0;
          for(const auto& r : gp.rows)
          {
            const double dx = x - r[0], dy = y - r[1], dz = z - r[2];
            s += r[4] * std::exp(-(dx * dx + dy * dy + dz * dz) / (2.0 * r[3] * r[3]));
          }
          return s;
        });
        Assembly::Common::ForceFunctional<decltype(f)> force(f);
        Assembly::assemble_linear_functional_vector(top.domain_assembler, vec_rhs, force, top.space, cubature_name);
      }
    }
    else
    {
      std::fprintf(stderr, "unknown --rhs %s\n", opt.rhs.c_str());
      return 2;
    }
    top.filter.filter_rhs(vec_rhs);
    const double setup_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_setup).count();

    // hierarchy: fine levels with Richardson(1) + Jacobi(omega) (or SOR / SSOR with the generic
    // backend), min = max = steps; coarse: exact inverse
    auto hierarchy = std::make_shared<Solver::MultiGridHierarchy<MatrixType, FilterType, TransferType>>(levels.size());
    for(std::size_t i = 0; (i + 1) < levels.size(); ++i)
    {
      LevelType& lvl = *levels.at(i);
      std::shared_ptr<Solver::SolverBase<VectorType>> precond;
      if(opt.smoother == "sor")
        precond = Solver::new_sor_precond(PreferredBackend::generic, lvl.matrix, lvl.filter, DataType(opt.sor_omega));
      else if(opt.smoother == "ssor")
        precond = Solver::new_ssor_precond(PreferredBackend::generic, lvl.matrix, lvl.filter, DataType(opt.sor_omega));
      else
        precond = Solver::new_jacobi_precond(lvl.matrix, lvl.filter, DataType(opt.omega));
      auto smoother = Solver::new_richardson(lvl.matrix, lvl.filter, DataType(1), precond);
      smoother->set_min_iter(opt.steps);
      smoother->set_max_iter(opt.steps);
      hierarchy->push_level(lvl.matrix, lvl.filter, lvl.transfer, smoother, smoother, smoother);
    }
    {
      LevelType& lvl = *levels.back();
      auto coarse = std::make_shared<CoarseInverseSolver>(lvl.matrix, lvl.filter);
      hierarchy->push_level(lvl.matrix, lvl.filter, coarse);
    }
    const Solver::MultiGridCycle cycle = opt.cycle == "f" ? Solver::MultiGridCycle::F :
                                         (opt.cycle == "w" ? Solver::MultiGridCycle::W : Solver::MultiGridCycle::V);
    auto multigrid = Solver::new_multigrid(hierarchy, cycle);
    if(opt.cgc == "energy")
      multigrid->set_adapt_cgc(Solver::MultiGridAdaptCGC::MinEnergy);
    else if(opt.cgc == "defect")
      multigrid->set_adapt_cgc(Solver::MultiGridAdaptCGC::MinDefect);
#ifdef FEAT_HAVE_CUDA
    // every LAFEM op from here on (smoother set-up, solve) goes to the CUDA backend: the library
    // (FEATB200_BACKEND builds, "b200") or FEAT's own GPU kernels ("cuda")
    if(opt.backend == "b200" || opt.backend == "cuda")
      Backend::set_preferred_backend(PreferredBackend::cuda);
#endif
#ifdef FEATB200_BACKEND
    std::shared_ptr<Solver::IterativeSolver<VectorType>> solver;
    if(opt.b200_solver)
      solver = std::make_shared<FEATB200::MultiGridPCG<MatrixType, FilterType, TransferType>>(hierarchy,
        double(opt.omega), int(opt.steps));
    else
      solver = Solver::new_pcg(top.matrix, top.filter, multigrid);
#else
    auto solver = Solver::new_pcg(top.matrix, top.filter, multigrid);
#endif
    solver->set_tol_rel(DataType(opt.tol));
    solver->set_max_iter(100);
    hierarchy->init();
    solver->init();

    const std::string& o = opt.out;
    if(opt.dump)
    {
      dump_vec(o + "/rhs.npy", vec_rhs);
      for(Index l = opt.level_min; l <= opt.level; ++l)
      {
        if(!opt.dump_levels && l != opt.level)
          continue;
        LevelType& lvl = *levels.at(std::size_t(opt.level - l));
        const std::string p = o + "/L" + std::to_string(l);
        dump_csr(p + "_A", lvl.matrix);
        const auto& fv = lvl.filter.get_filter_vector();
        std::vector<unsigned long long> idx(fv.indices(), fv.indices() + fv.used_elements());
        write_npy(p + "_filter_idx.npy", "<u8", 8, idx.data(), idx.size());
        write_npy(p + "_filter_val.npy", "<f8", 8, fv.elements(), fv.used_elements());
        const auto& vs = lvl.mesh.get_vertex_set();
        std::vector<double> xy;
        for(Index v = 0; v < vs.get_num_vertices(); ++v)
          for(int d = 0; d < dim_; ++d)
            xy.push_back(double(vs[v][d]));
        write_npy(p + "_coords.npy", "<f8", 8, xy.data(), xy.size());
        if(l > opt.level_min)
        {
          dump_csr(p + "_P", lvl.transfer.get_mat_prol());
          dump_csr(p + "_R", lvl.transfer.get_mat_rest());
        }
      }
    }

    // one V-cycle applied to the fine rhs
    if(opt.vcycle && opt.dump && !opt.b200_solver)
    {
      VectorType z = top.matrix.create_vector_r();
      multigrid->apply(z, vec_rhs);
      dump_vec(o + "/vcycle.npy", z);
    }

    // full solve
    VectorType vec_sol = top.matrix.create_vector_r();
    vec_sol.format();
    Solver::Status st = Solver::solve(*solver, vec_sol, vec_rhs, top.matrix, top.filter);
    const Index iters = solver->get_num_iter();
    const double def_init = double(solver->get_def_initial());
    const double def_final = double(solver->get_def_final());
    if(opt.dump)
      dump_vec(o + "/sol.npy", vec_sol);

    // iterates x_k and the recursive defect norms, by re-solving with max_iter = k
    std::vector<double> defs;
    if(opt.iterates > 0)
    {
      for(Index k = 1; k <= opt.iterates; ++k)
      {
        solver->set_max_iter(k);
        VectorType xk = top.matrix.create_vector_r();
        xk.format();
        Solver::solve(*solver, xk, vec_rhs, top.matrix, top.filter);
        defs.push_back(double(solver->get_def_final()));
        if(opt.dump)
          dump_vec(o + "/iterate_" + std::to_string(k) + ".npy", xk);
      }
      solver->set_max_iter(100);
      if(opt.dump)
        write_npy(o + "/defects.npy", "<f8", 8, defs.data(), defs.size());
    }

    // timing: one warm-up solve, then the median of REPS solves (solve only, no assembly)
    std::vector<double> times;
    for(int r = 0; r <= opt.time_reps && opt.time_reps > 0; ++r)
    {
      VectorType xs = top.matrix.create_vector_r();
      xs.format();
      auto t0 = std::chrono::steady_clock::now();
      Solver::solve(*solver, xs, vec_rhs, top.matrix, top.filter);
      auto t1 = std::chrono::steady_clock::now();
      if(r > 0)
        times.push_back(std::chrono::duration<double, std::milli>(t1 - t0).count());
    }
    double median = 0.0;
    std::string times_json = "[";
    for(std::size_t k = 0; k < times.size(); ++k)
      times_json += (k ? ", " : "") + std::to_string(times[k]);
    times_json += "]";
    if(!times.empty())
    {
      std::vector<double> sorted(times);
      std::sort(sorted.begin(), sorted.end());
      median = sorted[sorted.size() / 2];
    }

    solver->done();
    hierarchy->done();

    std::printf("{\"dim\": %d, \"level\": %lu, \"dofs\": %lu, \"nnz\": %lu, \"status\": \"%s\", \"iters\": %lu, "
      "\"def_init\": %.17g, \"def_final\": %.17g, \"setup_s\": %.3f, \"solve_ms_median\": %.6f, \"reps\": %zu, "
      "\"times_ms\": %s, \"backend\": \"%s\", \"solver\": \"%s\"}\n",
      dim_, (unsigned long)opt.level, (unsigned long)top.matrix.rows(), (unsigned long)top.matrix.used_elements(),
      Solver::status_success(st) ? "success" : "failure", (unsigned long)iters, def_init, def_final, setup_s,
      median, times.size(), times_json.c_str(), opt.backend.c_str(), opt.b200_solver ? "b200" : "feat");
    return 0;
  }
  // The reference's own solver test problem (kernel/solver/basic_solver-test.cpp:98-140): the
  // 5-point finite-difference matrix of PointstarFactoryFD(m, d), the Q2-bubble reference solution,
  // rhs = A * ref, and the iteration counts of the reference's CG and PCG-Jacobi from a zero guess.
  int run_fd(Index m, Index d, const std::string& out)
  {
    LAFEM::PointstarFactoryFD<DataType, IndexType> psf(m, d);
    MatrixType matrix(psf.matrix_csr());
    VectorType vec_ref(psf.vector_q2_bubble());
    VectorType vec_rhs = matrix.create_vector_r();
    matrix.apply(vec_rhs, vec_ref);
    LAFEM::NoneFilter<DataType, IndexType> filter;
    dump_csr(out + "/fd_A", matrix);
    dump_vec(out + "/fd_ref.npy", vec_ref);
    dump_vec(out + "/fd_rhs.npy", vec_rhs);
    Index iters[2];
    for(int k = 0; k < 2; ++k)
    {
      VectorType vec_sol = matrix.create_vector_r();
      vec_sol.format();
      std::shared_ptr<Solver::SolverBase<VectorType>> pre;
      if(k == 1)
        pre = Solver::new_jacobi_precond(matrix, filter);
      auto solver = Solver::new_pcg(matrix, filter, pre);
      solver->init();
      solver->apply(vec_sol, vec_rhs);
      iters[k] = solver->get_num_iter();
      solver->done();
      dump_vec(out + (k == 0 ? "/fd_sol_cg.npy" : "/fd_sol_pcgjac.npy"), vec_sol);
    }
    std::printf("{\"m\": %lu, \"d\": %lu, \"cg_iters\": %lu, \"pcg_jac_iters\": %lu}\n", (unsigned long)m,
      (unsigned long)d, (unsigned long)iters[0], (unsigned long)iters[1]);
    return 0;
  }
  // Container I/O round trip through the reference's own readers and writers: reads a binary CSR
  // matrix (fm_csr) and a binary dense vector (fm_dv), writes them back in the binary formats and
  // as Matrix Market / exponential ASCII into DIR (rt.csr, rt.dv, rt_matrix.mtx, rt_vector.mtx,
  // rt_vector.exp), and prints their sizes.
  int run_io(const char* csr_in, const char* dv_in, const std::string& out)
  {
    typedef LAFEM::SparseMatrixCSR<double, Index> MatrixType;
    typedef LAFEM::DenseVector<double, Index> VectorType;
    MatrixType a;
    a.read_from(LAFEM::FileMode::fm_csr, String(csr_in));
    VectorType v;
    v.read_from(LAFEM::FileMode::fm_dv, String(dv_in));
    a.write_out(LAFEM::FileMode::fm_csr, String(out + "/rt.csr"));
    v.write_out(LAFEM::FileMode::fm_dv, String(out + "/rt.dv"));
    a.write_out(LAFEM::FileMode::fm_mtx, String(out + "/rt_matrix.mtx"));
    v.write_out(LAFEM::FileMode::fm_mtx, String(out + "/rt_vector.mtx"));
    v.write_out(LAFEM::FileMode::fm_exp, String(out + "/rt_vector.exp"));
    std::printf("{\"rows\": %lu, \"columns\": %lu, \"used_elements\": %lu, \"size\": %lu}\n",
      (unsigned long)a.rows(), (unsigned long)a.columns(), (unsigned long)a.used_elements(),
      (unsigned long)v.size());
    return 0;
  }
} // namespace Oracle

int main(int argc, char* argv[])
{
  Runtime::ScopeGuard guard(argc, argv);
  Oracle::Options opt;
  if(argc == 5 && std::strcmp(argv[1], "fd") == 0)
    return Oracle::run_fd(Index(std::stoul(argv[2])), Index(std::stoul(argv[3])), argv[4]);
  if(argc == 5 && std::strcmp(argv[1], "io") == 0)
    return Oracle::run_io(argv[2], argv[3], argv[4]);
  if(argc < 2 || std::strcmp(argv[1], "solve") != 0)
  {
    std::fprintf(stderr, "usage: feat_oracle solve --dim D --level L --out DIR [...]\n");
    return 2;
  }
  for(int i = 2; i < argc; ++i)
  {
    std::string a = argv[i];
    auto next = [&](void) -> std::string
    {
      if(i + 1 >= argc)
      {
        std::fprintf(stderr, "missing value for %s\n", a.c_str());
        std::exit(2);
      }
      return std::string(argv[++i]);
    };
    if(a == "--dim") opt.dim = std::stoi(next());
    else if(a == "--level") opt.level = Index(std::stoul(next()));
    else if(a == "--level-min") opt.level_min = Index(std::stoul(next()));
    else if(a == "--out") opt.out = next();
    else if(a == "--rhs") opt.rhs = next();
    else if(a == "--params") opt.params = next();
    else if(a == "--kappa") opt.kappa = next();
    else if(a == "--omega") opt.omega = std::stod(next());
    else if(a == "--steps") opt.steps = Index(std::stoul(next()));
    else if(a == "--tol") opt.tol = std::stod(next());
    else if(a == "--iterates") opt.iterates = Index(std::stoul(next()));
    else if(a == "--vcycle") opt.vcycle = true;
    else if(a == "--cycle") opt.cycle = next();
    else if(a == "--cgc") opt.cgc = next();
    else if(a == "--dump-levels") opt.dump_levels = true;
    else if(a == "--no-dump") opt.dump = false;
    else if(a == "--time") opt.time_reps = std::stoi(next());
    else if(a == "--smoother") opt.smoother = next();
    else if(a == "--sor-omega") opt.sor_omega = std::stod(next());
#ifdef FEAT_HAVE_CUDA
    else if(a == "--backend") opt.backend = next();
#endif
#ifdef FEATB200_BACKEND
    else if(a == "--b200-solver") opt.b200_solver = true;
#endif
    else
    {
      std::fprintf(stderr, "unknown option %s\n", a.c_str());
      return 2;
    }
  }
  if(opt.dim == 2)
    return Oracle::run<2>(opt);
  if(opt.dim == 3)
    return Oracle::run<3>(opt);
  std::fprintf(stderr, "--dim must be 2 or 3\n");
  return 2;
}
