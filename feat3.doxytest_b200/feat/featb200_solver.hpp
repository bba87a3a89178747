// Solver-level binding for FEAT: PCG preconditioned by one multigrid cycle, run by libfeatb200.
//
// FEAT's own PCG + MultiGrid (kernel/solver/pcg.hpp:188-286, kernel/solver/multigrid.hpp:1270-2000)
// calls one backend op at a time; this class hands the whole solve to the library instead, which
// runs it as one device-resident CUDA graph.  It reads the levels of the same MultiGridHierarchy a
// FEAT application builds with push_level (multigrid.hpp:612-690) — system matrix, unit filter,
// transfer operator per level, finest first — and uploads them once in init_numeric().  Vectors
// may live in host or managed memory (FEAT's MemoryPool allocates managed memory in CUDA builds).
//
// The smoother must be what the library implements: Richardson(omega_R = 1) with Jacobi(omega)
// and min_iter == max_iter == steps on every level but the coarsest, an exact coarse solve; give
// omega and steps to the constructor (FEAT's smoother objects do not expose them).
#pragma once

#include <kernel/solver/iterative.hpp>
#include <kernel/solver/multigrid.hpp>
#include <kernel/util/exception.hpp>

#include <featb200.h>

#include <cstdint>
#include <memory>
#include <string>

namespace FEATB200
{
  // FEAT's Solver::Status for a library solver status (both follow kernel/solver/base.hpp:48-64)
  inline FEAT::Solver::Status to_feat_status(int st)
  {
    switch(st)
    {
      case FB_SOLVER_PROGRESS: return FEAT::Solver::Status::progress;
      case FB_SOLVER_SUCCESS: return FEAT::Solver::Status::success;
      case FB_SOLVER_ABORTED: return FEAT::Solver::Status::aborted;
      case FB_SOLVER_DIVERGED: return FEAT::Solver::Status::diverged;
      case FB_SOLVER_MAX_ITER: return FEAT::Solver::Status::max_iter;
      case FB_SOLVER_STAGNATED: return FEAT::Solver::Status::stagnated;
      default: return FEAT::Solver::Status::undefined;
    }
  }

  inline void check(fb_status st, const char* what)
  {
    if(st != FB_OK)
      throw FEAT::InternalError(what, __FILE__, __LINE__, std::string("libfeatb200: ") + fb_last_error());
  }

  template<typename Matrix_, typename Filter_, typename Transfer_>
  class MultiGridPCG :
    public FEAT::Solver::IterativeSolver<typename Matrix_::VectorTypeR>
  {
  public:
    typedef typename Matrix_::VectorTypeR VectorType;
    typedef FEAT::Solver::MultiGridHierarchy<Matrix_, Filter_, Transfer_> HierarchyType;
    typedef FEAT::Solver::IterativeSolver<VectorType> BaseClass;

  private:
    std::shared_ptr<HierarchyType> _hierarchy;
    fb_hierarchy* _h = nullptr;
    fb_solver* _s = nullptr;
    fb_solver_config _cfg;
    fb_solve_info _info;
    int _cap = 0;    // max_iter the device solver was created with

    static fb_csr_host view(const Matrix_& m)
    {
      static_assert(sizeof(typename Matrix_::IndexType) == sizeof(std::uint64_t), "64-bit FEAT::Index expected");
      return fb_csr_host{m.rows(), m.columns(), m.used_elements(),
                         reinterpret_cast<const std::uint64_t*>(m.row_ptr()),
                         reinterpret_cast<const std::uint64_t*>(m.col_ind()), m.val()};
    }

  public:
    // omega: the Jacobi damping; steps: the Richardson smoother's min_iter == max_iter
    MultiGridPCG(std::shared_ptr<HierarchyType> hierarchy, double omega, int steps) :
      BaseClass("B200-PCG-MG"), _hierarchy(hierarchy), _info()
    {
      fb_solver_config_default(&_cfg);
      _cfg.omega = omega;
      _cfg.smooth_steps = steps;
    }

    virtual ~MultiGridPCG() { release(); }

    virtual FEAT::String name() const override { return "B200-PCG-MG"; }

    // device choices (numbering, precision, cycle, ...) before init_numeric()
    fb_solver_config& config() { return _cfg; }

    virtual void init_numeric() override
    {
      BaseClass::init_numeric();
      release();
      const int nl = int(_hierarchy->size_physical());
      check(fb_hierarchy_create(&_h, nl), "fb_hierarchy_create");
      for(int l = 0; l < nl; ++l)
      {
        const auto& lvl = _hierarchy->get_level(FEAT::Index(l));
        const fb_csr_host A = view(lvl.get_system_matrix());
        const auto& fv = lvl.get_system_filter().get_filter_vector();
        const auto* fidx = reinterpret_cast<const std::uint64_t*>(fv.indices());
        const Transfer_* t = lvl.get_transfer_operator();
        if(l + 1 < nl)
        {
          const fb_csr_host P = view(t->get_mat_prol());
          const fb_csr_host R = view(t->get_mat_rest());
          check(fb_hierarchy_set_level(_h, l, &A, fidx, fv.elements(), fv.used_elements(), &P, &R),
                "fb_hierarchy_set_level");
        }
        else
          check(fb_hierarchy_set_level(_h, l, &A, fidx, fv.elements(), fv.used_elements(), nullptr, nullptr),
                "fb_hierarchy_set_level");
      }
      _cfg.tol_rel = double(this->_tol_rel);
      _cfg.tol_abs = double(this->_tol_abs);
      _cfg.max_iter = int(this->_max_iter);
      _cfg.min_iter = int(this->_min_iter);
      check(fb_solver_create(&_s, _h, &_cfg), "fb_solver_create");
      _cap = _cfg.max_iter;
    }

    virtual void done_numeric() override
    {
      release();
      BaseClass::done_numeric();
    }

    // PCG::correct semantics: vec_sol holds the initial guess on entry
    virtual FEAT::Solver::Status correct(VectorType& vec_sol, const VectorType& vec_rhs) override
    {
      if(_s == nullptr)
        throw FEAT::InternalError(__func__, __FILE__, __LINE__, "init_numeric() was not called");
      // tolerances and iteration limits set on the FEAT object after init_numeric()
      if(double(this->_tol_rel) != _cfg.tol_rel || double(this->_tol_abs) != _cfg.tol_abs)
      {
        _cfg.tol_rel = double(this->_tol_rel);
        _cfg.tol_abs = double(this->_tol_abs);
        check(fb_solver_set_tolerances(_s, _cfg.tol_rel, _cfg.tol_abs), "fb_solver_set_tolerances");
      }
      if(int(this->_max_iter) != _cfg.max_iter || int(this->_min_iter) != _cfg.min_iter)
      {
        if(int(this->_max_iter) > _cap)
          init_numeric();   // the device history holds the creation max_iter: build anew
        _cfg.max_iter = int(this->_max_iter);
        _cfg.min_iter = int(this->_min_iter);
        check(fb_solver_set_iteration_limits(_s, _cfg.min_iter, _cfg.max_iter), "fb_solver_set_iteration_limits");
      }
      check(fb_solver_solve(_s, vec_sol.elements(), vec_rhs.elements(), &_info), "fb_solver_solve");
      this->_num_iter = FEAT::Index(_info.iterations);
      this->_def_init = typename VectorType::DataType(_info.def_init);
      this->_def_cur = typename VectorType::DataType(_info.def_final);
      return to_feat_status(_info.status);
    }

    virtual FEAT::Solver::Status apply(VectorType& vec_cor, const VectorType& vec_def) override
    {
      vec_cor.format();
      return correct(vec_cor, vec_def);
    }

    // the solve's device time and kernel count (no FEAT counterpart)
    const fb_solve_info& info() const { return _info; }

  private:
    void release()
    {
      if(_s)
        fb_solver_destroy(_s);
      if(_h)
        fb_hierarchy_destroy(_h);
      _s = nullptr;
      _h = nullptr;
    }
  };
} // namespace FEATB200
