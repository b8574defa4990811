// Sample driver in the shape of the reference's Helmholtz-filter mains,
// written against include/icarat_b200.hpp: opt-mma-HelmholtzFilter
// (sample/algorithm/opt-mma-HelmholtzFilter/opt_mma_Helmholtz.cpp:86-170) and,
// with "oc", opt-macro-oc (sample/algorithm/opt-macro-oc/opt_macro_oc.cpp:
// 83-172).  Helmholtz density filter, threshold with beta =
// min(2^(step/40), 16), solve, compliance, volume constraint, sensitivity
// times the threshold derivative, the two sensitivity calls of the Helmholtz
// filter, then MMA, or OC whose volume functor filters each trial by the
// Helmholtz filter.
//
// usage: opt_mma_helmholtz <nx> <ny> <nz> <steps> <radius> [solver name] [mma|oc]
// (default "Eigen_LDLT", the MMA driver's choice at :99, and mma)
// prints "step <k> <compliance> <constraint> <cg iterations>" per iteration.
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
  if(argc < 6)
  {
    std::printf("usage: %s nx ny nz steps radius [solver name] [mma|oc]\n", argv[0]);
    return 1;
  }
  const int nx = std::atoi(argv[1]), ny = std::atoi(argv[2]), nz = std::atoi(argv[3]);
  const int steps = std::atoi(argv[4]);
  const double filterR = std::atof(argv[5]);
  const std::string solver = argc > 6 ? argv[6] : "Eigen_LDLT";
  const bool oc_update = argc > 7 && std::string(argv[7]) == "oc";
  try
  {
    // x = 0 face clamped, unit load at (nx, ny/2, 0)
    icarat_dirichlet clamp{{1, 1, 1}, {0, 0, 0}, {{0, 0}, {0, (double)ny}, {0, (double)nz}}};
    const double py = (double)(ny / 2);
    icarat_load load{{0, 0, -1.0}, {{(double)nx, (double)nx}, {py, py}, {0, 0}}};
    Model model(nx, ny, nz, nx, ny, nz, 1e-9, 1.0, 0.3, 3.0, {clamp}, {load});
    const int nelx = model.nelx;
    std::vector<double> design_s(nelx, 0.3), xmin(nelx, 1e-4), xmax(nelx, 1.0);
    std::vector<double> dfds, dgds;
    double vol = 0.0;
    check(icarat_element_stiffness(model.ctx(), nullptr, &vol), "element volume");
    FilterHelmholtz filter(model, filterR);
    LinearAnalysis compt(model);
    compt.tol = 1e-12;
    MMASolver mma(nelx, 1);
    mma.SetMoveLimit(0.2);
    OC oc(model, nelx);
    double V0 = 0.0;
    for(int optstep = 1; optstep <= steps; optstep++)
    {
      auto fil_s = filter.densityFilter(design_s, "Eigen_CG", 0, false);
      const double beta = std::min(std::pow(2.0, (int)(optstep / 40)), 16.0);
      auto thre_s = filter.threshold(fil_s, beta, 0.5);
      model.setDesignS(thre_s);
      compt.solve(solver, false);
      const double object_f = compt.compliance();
      double volume = 0.0;
      for(double v : thre_s)
        volume += v * vol;
      double const_h = 0.0;
      if(optstep == 1)
      {
        V0 = volume;
        const_h = oc_update ? V0 : 0.0;
      }
      else
        const_h = oc_update ? volume : volume / V0 - 1.0;
      compt.sensitivity(dfds, dgds, oc_update ? 1.0 : 1.0 / V0);
      auto thrediff = filter.thresholdDerivative(fil_s, beta, 0.5);
      for(int i = 0; i < nelx; i++)
      {
        dfds[i] *= thrediff[i];
        dgds[i] *= thrediff[i];
      }
      dfds = filter.densityFilter(dfds, "Eigen_CG", 0, true);
      dgds = filter.densityFilter(dgds, "Eigen_CG", 0, true);
      if(oc_update)
        oc.UpdateVariables(design_s, dfds, V0, dgds, xmin, xmax, true, beta, 0.5, true);
      else
        mma.Update(design_s.data(), dfds.data(), &const_h, dgds.data(), xmin.data(),
                   xmax.data());
      std::printf("step %d %.17g %.17g %d\n", optstep, object_f, const_h,
                  compt.info.iterations);
    }
  }
  catch(const Error &e)
  {
    std::printf("error %d: %s\n", e.status, e.what());
    return 2;
  }
  return 0;
}
