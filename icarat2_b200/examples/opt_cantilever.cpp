// Sample driver in the shape of the reference's opt-macro-mma-nondesign /
// opt-macro-oc mains (sample/algorithm/*/opt_macro_*.cpp), written against
// include/icarat_b200.hpp: same loop body, same call names, GPU underneath.
//
// usage: opt_cantilever <nx> <ny> <nz> <steps> <radius> <oc|mma> [MG_CG|Eigen_CG]
// prints "step <k> <compliance> <constraint> <cg iterations>" per design
// iteration.  The loop runs while Optimize::isConvergence(1e-5, 50) returns 1
// (opt_macro_oc.cpp:83,137), at most <steps> iterations, and prints
// "converged <k>" when the test ended it.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "icarat_b200.hpp"

using namespace icarat::b200;

int main(int argc, char **argv)
{
  if(argc < 7)
  {
    std::printf("usage: %s nx ny nz steps radius oc|mma [MG_CG|Eigen_CG]\n", argv[0]);
    return 1;
  }
  const int nx = std::atoi(argv[1]), ny = std::atoi(argv[2]), nz = std::atoi(argv[3]);
  const int steps = std::atoi(argv[4]);
  const double filterR = std::atof(argv[5]);
  const bool mma_update = std::string(argv[6]) == "mma";
  const std::string solver = argc > 7 ? argv[7] : "MG_CG";
  try
  {
    // [boundary_condition]: x = 0 face clamped, unit load at (nx, ny/2, 0)
    icarat_dirichlet clamp{{1, 1, 1}, {0, 0, 0}, {{0, 0}, {0, (double)ny}, {0, (double)nz}}};
    const double py = (double)(ny / 2);
    icarat_load load{{0, 0, -1.0}, {{(double)nx, (double)nx}, {py, py}, {0, 0}}};
    Model model(nx, ny, nz, nx, ny, nz, 1e-9, 1.0, 0.3, 3.0, {clamp}, {load});
    const int nelx = model.nelx;
    Optimize optim(nelx, 1, 1e-4, 1.0);
    std::vector<double> &design_s = optim.design_s, &xmin = optim.xmin, &xmax = optim.xmax;
    std::fill(design_s.begin(), design_s.end(), 0.3);
    std::vector<double> dfds, dgds;
    double vol = 0.0; // element volume (sum of det J w, elasticity.cpp:249)
    check(icarat_element_stiffness(model.ctx(), nullptr, &vol), "element volume");
    Filter filter(model, filterR);
    LinearAnalysis compt(model);
    compt.tol = 1e-12;
    MMASolver mma(nelx, 1);
    mma.SetMoveLimit(0.2);
    OC oc(model, nelx);
    double V0 = 0.0;
    int convergence = 1;
    while(convergence == 1 && optim.optstep < steps)
    {
      const int optstep = ++optim.optstep;
      auto design_filtered = filter.densityFilter(design_s, false);
      model.setDesignS(design_filtered);
      compt.solve(solver, false);
      const double object_f = compt.compliance();
      optim.object_f = object_f;
      double volume = 0.0;
      for(double v : design_filtered)
        volume += v * vol;
      double const_h;
      if(optstep == 1)
      {
        V0 = volume;
        const_h = mma_update ? 0.0 : V0;
      }
      else
        const_h = mma_update ? volume / V0 - 1.0 : volume;
      convergence = optim.isConvergence(1.0e-5, 50);
      compt.sensitivity(dfds, dgds, mma_update ? 1.0 / V0 : 1.0);
      dfds = filter.densityFilter(dfds, true);
      dgds = filter.densityFilter(dgds, true);
      if(mma_update)
        mma.Update(design_s.data(), dfds.data(), &const_h, dgds.data(), xmin.data(),
                   xmax.data());
      else
        oc.UpdateVariables(design_s, dfds, V0, dgds, xmin, xmax);
      std::printf("step %d %.17g %.17g %d\n", optstep, object_f, const_h,
                  compt.info.iterations);
    }
    if(convergence == 0)
      std::printf("converged %d\n", optim.optstep);
  }
  catch(const Error &e)
  {
    std::printf("error %d: %s\n", e.status, e.what());
    return 2;
  }
  return 0;
}
