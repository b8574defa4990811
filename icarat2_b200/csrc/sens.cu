// Post-solve element quantities: nodal values, compliance and the compliance
// sensitivity of the sample drivers.
#include <cmath>

#include "stencil.cuh"

namespace icarat_b200
{

// divideValIntoNode (src/analysis/analysis_utility.hpp:9-31): free values from
// the solution, prescribed values on constrained components, |v| < 1e-15 -> 0.
__device__ __forceinline__ double node_value(const double *__restrict__ u,
                                             const double *__restrict__ uD,
                                             unsigned fix, long id, int q)
{
  double v = ((fix >> q) & 1u) ? (uD ? uD[id] : 0.0) : u[id];
  return fabs(v) < 1.0e-15 ? 0.0 : v;
}

__global__ void k_node_values(int numnp, const double *__restrict__ u,
                              const double *__restrict__ uD,
                              const uint8_t *__restrict__ fix,
                              double *__restrict__ out)
{
  for(int n = blockIdx.x * blockDim.x + threadIdx.x; n < numnp;
      n += gridDim.x * blockDim.x)
  {
    const unsigned f = fix[n];
#pragma unroll
    for(int q = 0; q < 3; q++)
      out[3L * n + q] = node_value(u, uD, f, (long)q * numnp + n, q);
  }
}

// Driver sensitivity() (sample/algorithm/opt-macro-oc/opt_macro_oc.cpp:182-212):
//   young  = (1 - rho^p) E1 + rho^p E2,  dyoung = p rho^(p-1) (E2 - E1)
//   dfds_e = -(dyoung / young) u_e^T (young Ke0) u_e,   dgds_e = volume * scale
// with u_e the truncated nodal values.
__global__ void __launch_bounds__(128)
    k_sensitivity(GridDev g, KeParam ke, const double *__restrict__ rho,
                  const double *__restrict__ u, const double *__restrict__ uD,
                  const uint8_t *__restrict__ fix, double e1, double e2, double p,
                  double vol, double scale, double *__restrict__ dfds,
                  double *__restrict__ dgds)
{
  for(int e = blockIdx.x * blockDim.x + threadIdx.x; e < g.nelx;
      e += gridDim.x * blockDim.x)
  {
    const int i = e % g.nx, j = (e / g.nx) % g.ny, k = e / (g.nx * g.ny);
    double ue[24];
#pragma unroll
    for(int bz = 0; bz < 2; bz++)
#pragma unroll
      for(int by = 0; by < 2; by++)
#pragma unroll
        for(int bx = 0; bx < 2; bx++)
        {
          const int b = local_node(bx, by, bz);
          const long m = (i + bx) + (long)(j + by) * g.NX + (long)(k + bz) * g.NX * g.NY;
          const unsigned f = fix[m];
#pragma unroll
          for(int q = 0; q < 3; q++)
            ue[3 * b + q] = node_value(u, uD, f, (long)q * g.numnp + m, q);
        }
    const double dens = rho[e];
    const double young = (1.0 - pow(dens, p)) * e1 + pow(dens, p) * e2;
    const double dyoung = p * pow(dens, p - 1.0) * (e2 - e1);
    double q = 0.0;
#pragma unroll
    for(int r = 0; r < 24; r++)
    {
      double s = 0.0;
#pragma unroll
      for(int c = 0; c < 24; c++)
        s = fma(ke.k[24 * r + c], ue[c], s);
      q = fma(ue[r], s, q);
    }
    if(dfds)
      dfds[e] = -(dyoung / young) * (young * q);
    if(dgds)
      dgds[e] = vol * scale;
  }
}

// von Mises stress of the last solve per element (Elastic::makeMisesStress,
// src/problem/elasticity.cpp:166-207): sigma = E(rho) S u_e with the
// Gauss-averaged stress operator S and the truncated nodal values,
// mises = sqrt(sigma^T V sigma), V = [1 -1/2 -1/2; ..] (+) 3 I on the shears
__global__ void __launch_bounds__(128)
    k_mises(GridDev g, StressParam sp, const double *__restrict__ rho,
            const double *__restrict__ u, const double *__restrict__ uD,
            const uint8_t *__restrict__ fix, double e1, double e2, double p,
            double *__restrict__ out)
{
  for(int e = blockIdx.x * blockDim.x + threadIdx.x; e < g.nelx;
      e += gridDim.x * blockDim.x)
  {
    const int i = e % g.nx, j = (e / g.nx) % g.ny, k = e / (g.nx * g.ny);
    double ue[24];
#pragma unroll
    for(int bz = 0; bz < 2; bz++)
#pragma unroll
      for(int by = 0; by < 2; by++)
#pragma unroll
        for(int bx = 0; bx < 2; bx++)
        {
          const int b = local_node(bx, by, bz);
          const long m = (i + bx) + (long)(j + by) * g.NX + (long)(k + bz) * g.NX * g.NY;
          const unsigned f = fix[m];
#pragma unroll
          for(int q = 0; q < 3; q++)
            ue[3 * b + q] = node_value(u, uD, f, (long)q * g.numnp + m, q);
        }
    const double dens = rho[e];
    const double young = (1.0 - pow(dens, p)) * e1 + pow(dens, p) * e2;
    double sg[6];
#pragma unroll
    for(int r = 0; r < 6; r++)
    {
      double t = 0.0;
#pragma unroll
      for(int c = 0; c < 24; c++)
        t = fma(sp.s[24 * r + c], ue[c], t);
      sg[r] = young * t;
    }
    const double q = sg[0] * (sg[0] - 0.5 * sg[1] - 0.5 * sg[2]) +
                     sg[1] * (sg[1] - 0.5 * sg[0] - 0.5 * sg[2]) +
                     sg[2] * (sg[2] - 0.5 * sg[0] - 0.5 * sg[1]) +
                     3.0 * (sg[3] * sg[3] + sg[4] * sg[4] + sg[5] * sg[5]);
    out[e] = sqrt(fmax(q, 0.0)); // V is positive semidefinite: q < 0 is rounding
  }
}

void mises_dev(icarat_ctx *c, double *out)
{
  IREQUIRE(c->solved, ICARAT_ERR_STATE, "Mises stress needs a solve first");
  GridDev g{c->nx, c->ny, c->nz, c->NX, c->NY, c->NZ, c->numnp, c->nelx};
  note_launch();
  k_mises<<<(c->nelx + 127) / 128, 128, 0, c->stream>>>(g, c->sb0, c->d_rho, c->d_u, c->d_uD,
                                                        c->d_fix, c->mat.young_min,
                                                        c->mat.young_max, c->mat.penalty, out);
  ICK(cudaGetLastError());
}

void node_values_dev(icarat_ctx *c, double *out)
{
  note_launch();
  k_node_values<<<(c->numnp + 255) / 256, 256, 0, c->stream>>>(c->numnp, c->d_u,
                                                               c->d_uD, c->d_fix, out);
  ICK(cudaGetLastError());
}

double compliance_dev(icarat_ctx *c)
{
  return device_dot(c, c->d_u, c->d_fext, c->neq);
}

void sensitivity_dev(icarat_ctx *c, double scale, double *dfds, double *dgds)
{
  IREQUIRE(c->solved, ICARAT_ERR_STATE, "sensitivity needs a solve first");
  GridDev g{c->nx, c->ny, c->nz, c->NX, c->NY, c->NZ, c->numnp, c->nelx};
  note_launch();
  k_sensitivity<<<(c->nelx + 127) / 128, 128, 0, c->stream>>>(
      g, c->ke0, c->d_rho, c->d_u, c->d_uD, c->d_fix, c->mat.young_min,
      c->mat.young_max, c->mat.penalty, c->vol0, scale, dfds, dgds);
  ICK(cudaGetLastError());
}

} // namespace icarat_b200
