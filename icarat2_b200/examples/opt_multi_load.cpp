// Sample driver in the shape of the reference's opt-multi-load main
// (sample/software/opt-multi-load/opt_multi_load.cpp:86-200) on the voxel
// box, through the C ABI's device-resident loop: the load cases go in as
// icarat_set_load_cases (the vector<Force> of :68-80), the design /
// non-design IDs of getDesignNonDesignIDs (src/misc/non_design_domain.hpp)
// as icarat_loop_set_domains, the Helmholtz filter (filterR) and threshold
// as loop options; each icarat_loop_step solves every case on the design,
// sums compliances and sensitivities, filters, zeroes the non-design
// sensitivities and updates by MMA.
//
// usage: opt_multi_load <nx> <ny> <nz> <steps> <filterR>
// cases: tip down at (nx, ny/2, 0), tip sideways at (nx, ny, nz), tip up at
// (nx, 0, nz); non-design: the two element columns next to the loaded face.
// prints "step <k> <compliance sum> <constraint> <cg iterations>".
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "icarat_b200.hpp"

using namespace icarat::b200;

int main(int argc, char **argv)
{
  if(argc < 6)
  {
    std::printf("usage: %s nx ny nz steps filterR\n", argv[0]);
    return 1;
  }
  const int nx = std::atoi(argv[1]), ny = std::atoi(argv[2]), nz = std::atoi(argv[3]);
  const int steps = std::atoi(argv[4]);
  const double filterR = std::atof(argv[5]);
  try
  {
    icarat_dirichlet clamp{{1, 1, 1}, {0, 0, 0}, {{0, 0}, {0, (double)ny}, {0, (double)nz}}};
    const double X = nx, Y = ny, Z = nz, py = (double)(ny / 2);
    const icarat_load cases[3] = {{{0, 0, -1.0}, {{X, X}, {py, py}, {0, 0}}},
                                  {{0, -1.0, 0}, {{X, X}, {Y, Y}, {Z, Z}}},
                                  {{0, 0, 1.0}, {{X, X}, {0, 0}, {Z, Z}}}};
    // the force vector of each case (BCIcarat::input_neumann per case)
    std::vector<double> fext;
    int numeq = 0;
    for(const icarat_load &l : cases)
    {
      Model m(nx, ny, nz, nx, ny, nz, 1e-9, 1.0, 0.3, 3.0, {clamp}, {l});
      numeq = m.numeq;
      std::vector<double> f(numeq);
      check(icarat_fext(m.ctx(), f.data()), "fext");
      fext.insert(fext.end(), f.begin(), f.end());
    }
    Model model(nx, ny, nz, nx, ny, nz, 1e-9, 1.0, 0.3, 3.0, {clamp}, {cases[0]});
    const int nelx = model.nelx;
    icarat_loop_opts o{};
    o.method = 1; // MMA
    o.use_threshold = 1;
    o.T = 0.5;
    o.move = 0.2;
    o.xmin = 1.0e-4;
    o.xmax = 1.0;
    o.filter_radius = filterR;
    o.filter_kind = 1; // FilterHelmholtz
    o.solve = icarat_solve_opts{ICARAT_SOLVER_MG_PCG, 1.0e-12, 10000, 3, 2, 0, 0.0};
    std::vector<double> x0(nelx, 0.3);
    check(icarat_loop_init(model.ctx(), &o, x0.data()), "loop_init");
    check(icarat_set_load_cases(model.ctx(), 3, fext.data()), "set_load_cases");
    // non-design: elements with i >= nx - 2; design: the rest (set difference)
    std::vector<int> design, nondesign;
    for(int e = 0; e < nelx; e++)
      (e % nx >= nx - 2 ? nondesign : design).push_back(e);
    check(icarat_loop_set_domains(model.ctx(), design.data(), (int)design.size(),
                                  nondesign.data(), (int)nondesign.size()),
          "loop_set_domains");
    for(int k = 1; k <= steps; k++)
    {
      icarat_step_info info{};
      check(icarat_loop_step(model.ctx(), &info), "loop_step");
      std::printf("step %d %.17g %.17g %d\n", k, info.compliance, info.constraint,
                  info.cg_iterations);
    }
  }
  catch(const Error &e)
  {
    std::printf("error %d: %s\n", e.status, e.what());
    return 2;
  }
  return 0;
}
