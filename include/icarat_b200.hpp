// icarat_b200.hpp -- header-only C++ layer over icarat_gpu.h that keeps the
// reference's class names, method names and argument meanings for the
// linear-static SIMP path, so a sample-style main() switches by changing its
// includes and constructor arguments:
//
//   reference (src/...)                          this header
//   MeshIcarat + BCIcarat (io/*.hpp)        ->   icarat::b200::Model
//   LinearAnalysis<E,N>::solve(name, log)   ->   icarat::b200::LinearAnalysis::solve
//   Filter<E,N>::densityFilter(x, isSens)   ->   icarat::b200::Filter::densityFilter
//   Filter::threshold / thresholdDerivative ->   same names
//   OC::UpdateVariables(x, df, g, dg, ...)  ->   icarat::b200::OC::UpdateVariables
//   MMASolver::Update(x, df, g, dg, ...)    ->   icarat::b200::MMASolver::Update
//   Optimize::isConvergence(eps, minstep)    ->   icarat::b200::Optimize::isConvergence
//
// Errors: the reference prints and calls exit(1) (solvers.cpp:59,
// filter.hpp:130-134); here every failing call throws icarat::b200::Error with
// the library status and message.
#pragma once
#include <cmath>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

#include "icarat_gpu.h"

namespace icarat
{
namespace b200
{

struct Error : std::runtime_error
{
  int status;
  Error(int s, const std::string &what)
      : std::runtime_error(what + ": " + icarat_last_error()), status(s)
  {
  }
};

inline int check(int status, const char *what)
{
  if(status < 0)
    throw Error(status, what);
  return status;
}

struct Box
{
  double lo[3], hi[3];
};

// [mesh] + [material] + [boundary_condition] of a voxel box
class Model
{
public:
  Model(int nx, int ny, int nz, double lx, double ly, double lz, double young_min,
        double young_max, double poisson, double penalty,
        const std::vector<icarat_dirichlet> &dirichlet,
        const std::vector<icarat_load> &loads, int device = 0)
  {
    icarat_grid g{nx, ny, nz, lx, ly, lz};
    icarat_material m{young_min, young_max, poisson, penalty};
    icarat_bc bc{(int)dirichlet.size(), dirichlet.data(), (int)loads.size(),
                 loads.data()};
    check(icarat_ctx_create(&g, &m, &bc, device, &ctx_), "icarat_ctx_create");
    check(icarat_sizes(ctx_, &numnp, &nelx, &neq, &numeq), "icarat_sizes");
  }
  ~Model() { icarat_ctx_destroy(ctx_); }
  Model(const Model &) = delete;
  Model &operator=(const Model &) = delete;

  icarat_ctx *ctx() const { return ctx_; }
  // element[i].setDesignS(design_s[i]) for all elements
  void setDesignS(const std::vector<double> &design_s)
  {
    check(icarat_set_design(ctx_, design_s.data()), "setDesignS");
  }
  std::vector<double> fext() const
  {
    std::vector<double> f(numeq);
    check(icarat_fext(ctx_, f.data()), "fext");
    return f;
  }

  int numnp = 0, nelx = 0, neq = 0, numeq = 0;

private:
  icarat_ctx *ctx_ = nullptr;
};

// Optimize (src/optimization/opt_base.hpp:14-76): the design state of a
// sample driver's loop and its convergence test.  object_old, which the
// reference leaves uninitialised, starts at 0.
class Optimize
{
public:
  Optimize(int design, int constraint, double xmin_, double xmax_)
      : design_s(design), const_h(constraint), dfds(design),
        dgds((size_t)constraint * design), xmin(design, xmin_), xmax(design, xmax_)
  {
  }
  // 0 when |object_old - object_f| / object_f < epsilon and optstep >
  // minstep, else 1 with object_old = object_f
  int isConvergence(double epsilon, double minstep)
  {
    if(std::fabs(object_old - object_f) / object_f < epsilon && optstep > minstep)
      return 0;
    object_old = object_f;
    return 1;
  }

  std::vector<double> design_s, const_h, dfds, dgds, xmin, xmax;
  int optstep = 0;
  double object_f = 0.0;

private:
  double object_old = 0.0;
};

// LinearAnalysis<LinearElastic, Node> (src/analysis/linear.hpp:15-41)
class LinearAnalysis
{
public:
  explicit LinearAnalysis(Model &m) : m_(m), val(m.numeq) {}
  // solvName: "Eigen_CG" / "Scaling_CG" / "CG" (Jacobi-PCG), "MG_CG"
  // (multigrid), "Mixed_MG_CG" (FP32 multigrid-PCG refined by FP64
  // residuals); the reference's other names (Solvers::solve,
  // solvers.cpp:27-61) run multigrid-PCG: "ICCG", "Eigen_ICCG",
  // "Eigen_BiCGSTAB" at tol, the direct "Eigen_SparseLU", "Eigen_LDLT",
  // "Pardiso_*" to 1e-12
  void solve(const std::string &solvName, bool log)
  {
    icarat_solve_opts o{ICARAT_SOLVER_JACOBI_PCG, tol, maxIter, mg_levels, mg_smooth, 0, 0.0};
    static const char *direct[] = {"Eigen_SparseLU", "Eigen_LDLT", "Pardiso_LDLT",
                                   "Pardiso_LLT", "Pardiso_LU"};
    bool is_direct = false;
    for(const char *d : direct)
      is_direct = is_direct || solvName == d;
    if(solvName == "MG_CG" || solvName == "ICCG" || solvName == "Eigen_ICCG" ||
       solvName == "Eigen_BiCGSTAB" || is_direct)
      o.method = ICARAT_SOLVER_MG_PCG;
    else if(solvName == "Mixed_MG_CG")
      o.method = ICARAT_SOLVER_MIXED_IR;
    else if(solvName != "Eigen_CG" && solvName != "Scaling_CG" && solvName != "CG")
      throw Error(ICARAT_ERR_UNSUPPORTED, "Solver type name is wrong: " + solvName);
    if(is_direct && o.rtol > 1e-12)
      o.rtol = 1e-12;
    check(icarat_solve(m_.ctx(), &o, val.data(), &info), "LinearAnalysis::solve");
    if(log)
      printf("iteration: %d\nresidual: %g\n", info.iterations, info.rel_residual);
  }
  // object_f = value.val . fext
  double compliance() const
  {
    double c = 0.0;
    check(icarat_compliance(m_.ctx(), &c), "compliance");
    return c;
  }
  // node.val of every node after divideValIntoNode (numnp x 3)
  std::vector<double> nodeValues() const
  {
    std::vector<double> v(3 * (size_t)m_.numnp);
    check(icarat_node_values(m_.ctx(), v.data()), "nodeValues");
    return v;
  }
  // the sample drivers' sensitivity(): dfds, dgds (= volume * dgds_scale)
  void sensitivity(std::vector<double> &dfds, std::vector<double> &dgds,
                   double dgds_scale = 1.0) const
  {
    dfds.resize(m_.nelx);
    dgds.resize(m_.nelx);
    check(icarat_sensitivity(m_.ctx(), dgds_scale, dfds.data(), dgds.data()),
          "sensitivity");
  }

  double tol = 1.0e-10; // solvers.hpp:89
  int maxIter = 10000;  // solvers.hpp:90
  int mg_levels = 4, mg_smooth = 2;
  std::vector<double> val; // Value::val
  icarat_solve_info info{};

private:
  Model &m_;
};

// Filter<E,N> (src/optimization/filter.hpp:17-61)
class Filter
{
public:
  Filter(Model &m, double radius) : m_(m)
  {
    check(icarat_filter_setup(m.ctx(), radius), "Filter");
  }
  std::vector<double> densityFilter(const std::vector<double> &design_s, bool isSens)
  {
    std::vector<double> out(m_.nelx);
    check(icarat_density_filter(m_.ctx(), design_s.data(), out.data(), isSens ? 1 : 0),
          "densityFilter");
    return out;
  }
  std::vector<double> sensitivityFilter(const std::vector<double> &design_s,
                                        const std::vector<double> &dfds)
  {
    std::vector<double> out(m_.nelx);
    check(icarat_sensitivity_filter(m_.ctx(), design_s.data(), dfds.data(), out.data()),
          "sensitivityFilter");
    return out;
  }
  std::vector<double> threshold(const std::vector<double> &d, double beta, double T)
  {
    std::vector<double> out(m_.nelx);
    check(icarat_threshold(m_.ctx(), d.data(), beta, T, out.data()), "threshold");
    return out;
  }
  std::vector<double> thresholdDerivative(const std::vector<double> &d, double beta,
                                          double T)
  {
    std::vector<double> out(m_.nelx);
    check(icarat_threshold_derivative(m_.ctx(), d.data(), beta, T, out.data()),
          "thresholdDerivative");
    return out;
  }

private:
  Model &m_;
};

// FilterHelmholtz<E,N> (src/optimization/filter_helm.hpp:16-65): the nodal
// Helmholtz system solved on the GPU by Jacobi-PCG to 1e-10 for any of the
// reference's solver names (a well-conditioned mass + diffusion system: the
// name selects nothing else); unknown names throw as Solvers::solve exits
class FilterHelmholtz
{
public:
  FilterHelmholtz(Model &m, double radious) : m_(m)
  {
    check(icarat_helmholtz_setup(m.ctx(), radious), "FilterHelmholtz");
  }
  std::vector<double> densityFilter(const std::vector<double> &design_s,
                                    const std::string &solvName, int log, bool sensFlag)
  {
    static const char *names[] = {"Eigen_CG", "Scaling_CG", "CG", "ICCG", "Eigen_ICCG",
                                  "Eigen_BiCGSTAB", "Eigen_SparseLU", "Eigen_LDLT",
                                  "Pardiso_LDLT", "Pardiso_LLT", "Pardiso_LU"};
    bool known = false;
    for(const char *nm : names)
      known = known || solvName == nm;
    if(!known)
      throw Error(ICARAT_ERR_UNSUPPORTED, "Solver type name is wrong: " + solvName);
    std::vector<double> out(m_.nelx);
    icarat_solve_info info{};
    check(icarat_helmholtz_filter(m_.ctx(), design_s.data(), out.data(), sensFlag ? 1 : 0,
                                  0.0, 0, &info),
          "densityFilter");
    if(log == 1)
      std::printf("Helmholtz filtering...\n#iterations:     %d\nestimated error: %g\n",
                  info.iterations, info.rel_residual);
    return out;
  }
  std::vector<double> threshold(const std::vector<double> &d, double beta, double T)
  {
    std::vector<double> out(m_.nelx);
    check(icarat_threshold(m_.ctx(), d.data(), beta, T, out.data()), "threshold");
    return out;
  }
  std::vector<double> thresholdDerivative(const std::vector<double> &d, double beta,
                                          double T)
  {
    std::vector<double> out(m_.nelx);
    check(icarat_threshold_derivative(m_.ctx(), d.data(), beta, T, out.data()),
          "thresholdDerivative");
    return out;
  }

private:
  Model &m_;
};

// OC (src/optimization/opt-solver/OCSolver.hpp:13-80).  The reference takes
// the volume functor as a lambda; here it is the sample drivers' functor,
// g(x) = sum thr(filter(x)) v, evaluated on the GPU with the Model's Filter
// (threshold on when useThreshold is set).
class OC
{
public:
  OC(Model &m, int n) : m_(m), n_(n) {}
  void setMoveLimit(double mv) { movelimit = mv; }
  void UpdateVariables(std::vector<double> &xk, std::vector<double> &dfdx, double g,
                       std::vector<double> &dgdx, std::vector<double> &xmin,
                       std::vector<double> &xmax, bool useThreshold = false,
                       double beta = 1.0, double T = 0.5, bool helmholtz = false)
  {
    // helmholtz: the volume functor filters by FilterHelmholtz, as
    // opt_macro_oc.cpp:153-164 does
    icarat_oc_opts o{movelimit, 0.5, 0.0, 1.0e4, 1.0e-5, 100, useThreshold ? 1 : 0,
                     beta, T, helmholtz ? 1 : 0};
    int steps = 0;
    check(icarat_oc_update(m_.ctx(), xk.data(), dfdx.data(), g, dgdx.data(), xmin.data(),
                           xmax.data(), &o, &steps),
          "OC::UpdateVariables");
    (void)n_;
  }

private:
  Model &m_;
  int n_;
  double movelimit = 0.15;
};

// MMASolver (src/optimization/opt-solver/MMASolver.hpp:62-116)
class MMASolver
{
public:
  MMASolver(int n, int m, double a = 0.0, double c = 100000.0, double d = 0.0,
            int device = 0)
  {
    check(icarat_mma_create(device, n, m, a, c, d, &h_), "MMASolver");
  }
  ~MMASolver() { icarat_mma_destroy(h_); }
  MMASolver(const MMASolver &) = delete;
  MMASolver &operator=(const MMASolver &) = delete;
  void SetAsymptotes(double init, double decrease, double increase)
  {
    check(icarat_mma_set_asymptotes(h_, init, decrease, increase), "SetAsymptotes");
  }
  void SetMoveLimit(double m) { check(icarat_mma_set_move_limit(h_, m), "SetMoveLimit"); }
  void SetOscillation(double a)
  {
    check(icarat_mma_set_oscillation(h_, a), "SetOscillation");
  }
  void Update(double *xval, const double *dfdx, const double *gx, const double *dgdx,
              const double *xmin, const double *xmax)
  {
    check(icarat_mma_update(h_, xval, dfdx, gx, dgdx, xmin, xmax), "MMASolver::Update");
  }

private:
  icarat_mma *h_ = nullptr;
};

} // namespace b200
} // namespace icarat
