// C entry points over the reference's own MMASolver and OC classes, compiled
// from the reference sources by oracle/Makefile into oracle/_ref/.
// TEST INFRASTRUCTURE ONLY: used by tests/ to pin the oracle's MMA and OC
// restatements against the reference implementation.
#include <algorithm>
#include <cmath>
#include <iostream>
#include <vector>
#include "optimization/opt-solver/MMASolver.hpp"
#include "optimization/opt-solver/OCSolver.hpp"

extern "C" {

void *ref_mma_create(int n, int m, double a, double c, double d)
{
  return new icarat::MMASolver(n, m, a, c, d);
}
void ref_mma_destroy(void *p) { delete static_cast<icarat::MMASolver *>(p); }
void ref_mma_set_move(void *p, double mv)
{
  static_cast<icarat::MMASolver *>(p)->SetMoveLimit(mv);
}
void ref_mma_set_asymptotes(void *p, double i, double d, double c)
{
  static_cast<icarat::MMASolver *>(p)->SetAsymptotes(i, d, c);
}
void ref_mma_set_oscillation(void *p, double a)
{
  static_cast<icarat::MMASolver *>(p)->SetOscillation(a);
}
void ref_mma_update(void *p, double *x, const double *dfdx, const double *gx,
                    const double *dgdx, const double *xmin, const double *xmax)
{
  static_cast<icarat::MMASolver *>(p)->Update(x, dfdx, gx, dgdx, xmin, xmax);
}

typedef double (*ref_volume_fn)(const double *x, int n, void *user);

// OC::UpdateVariables with a C volume callback standing in for the driver's
// lambda.
void ref_oc_update(int n, double *x, double *dfdx, double g, double *dgdx,
                   const double *xmin, const double *xmax, double move,
                   ref_volume_fn fn, void *user)
{
  icarat::OC oc(n);
  oc.setMoveLimit(move);
  std::vector<double> xv(x, x + n), df(dfdx, dfdx + n), dg(dgdx, dgdx + n),
      mn(xmin, xmin + n), mx(xmax, xmax + n);
  oc.UpdateVariables(xv, df, g, dg, mn, mx,
                     [&](std::vector<double> &xk)
                     { return fn(xk.data(), n, user); });
  std::copy(xv.begin(), xv.end(), x);
}
}
