// Per-node FP64 stiffness stencil shared by the operator kernels.
//
// (K u)_n = sum_{e containing n} E_e Ke0[rows of n in e] u_e, evaluated by
// node ownership: the thread of node n gathers the 27 nodal displacements
// around it and the moduli of its (up to) 8 elements, so no two threads
// write the same output and no atomics or colouring are needed.  Ke0 is a
// by-value kernel parameter; after full unrolling every coefficient is a
// constant-bank operand of a DFMA (576 per node).
#pragma once
#include "internal.cuh"

namespace icarat_b200
{

// local node number of the corner (lx, ly, lz) of a hexa8
// (mesh_icarat.hpp:489-509 order)
__host__ __device__ constexpr int local_node(int lx, int ly, int lz)
{
  return 4 * lz + (ly ? (lx ? 2 : 3) : (lx ? 1 : 0));
}

// One z-layer of 4 elements around node (i,j,k): SZ = 0 are the elements
// below the node (element k index k-1), SZ = 1 the ones above.  ul[bz][s]
// holds the displacements of node layer k - 1 + SZ + bz, s = (dy+1)*3+(dx+1).
template <int SZ>
__device__ __forceinline__ void layer_contrib(const KeParam &ke,
                                              const double (&ul)[2][9][3],
                                              const double (&Ev)[4],
                                              double (&acc)[3])
{
#pragma unroll
  for(int sy = 0; sy < 2; sy++)
#pragma unroll
    for(int sx = 0; sx < 2; sx++)
    {
      const int a = local_node(1 - sx, 1 - sy, 1 - SZ);
      double t0 = 0.0, t1 = 0.0, t2 = 0.0;
#pragma unroll
      for(int bz = 0; bz < 2; bz++)
#pragma unroll
        for(int by = 0; by < 2; by++)
#pragma unroll
          for(int bx = 0; bx < 2; bx++)
          {
            const int b = local_node(bx, by, bz);
            const int s = (sy + by) * 3 + (sx + bx);
#pragma unroll
            for(int d = 0; d < 3; d++)
            {
              const double u = ul[bz][s][d];
              t0 = fma(ke.k[(3 * a + 0) * 24 + 3 * b + d], u, t0);
              t1 = fma(ke.k[(3 * a + 1) * 24 + 3 * b + d], u, t1);
              t2 = fma(ke.k[(3 * a + 2) * 24 + 3 * b + d], u, t2);
            }
          }
      const double e = Ev[sy * 2 + sx];
      acc[0] = fma(e, t0, acc[0]);
      acc[1] = fma(e, t1, acc[1]);
      acc[2] = fma(e, t2, acc[2]);
    }
}

__device__ __forceinline__ void load_layer(const double *__restrict__ u,
                                           const GridDev &g, int i, int j,
                                           int kk, double (&L)[9][3])
{
  const bool kin = kk >= 0 && kk < g.NZ;
#pragma unroll
  for(int dy = -1; dy <= 1; dy++)
#pragma unroll
    for(int dx = -1; dx <= 1; dx++)
    {
      const int ii = i + dx, jj = j + dy;
      const bool in = kin && ii >= 0 && ii < g.NX && jj >= 0 && jj < g.NY;
      const long m = (long)ii + (long)jj * g.NX + (long)kk * g.NX * g.NY;
      const int s = (dy + 1) * 3 + (dx + 1);
#pragma unroll
      for(int d = 0; d < 3; d++)
        L[s][d] = in ? __ldg(u + 3 * m + d) : 0.0;
    }
}

__device__ __forceinline__ double load_E(const double *__restrict__ E,
                                         const GridDev &g, int ei, int ej,
                                         int ek)
{
  const bool in = ei >= 0 && ei < g.nx && ej >= 0 && ej < g.ny && ek >= 0 &&
                  ek < g.nz;
  return in ? __ldg(E + ei + (long)ej * g.nx + (long)ek * g.nx * g.ny) : 0.0;
}

// (K u) at node n (unmasked) and the node's own displacement uc.
__device__ __forceinline__ void node_Ku(const GridDev &g, const KeParam &ke,
                                        const double *__restrict__ E,
                                        const double *__restrict__ u, int n,
                                        double (&acc)[3], double (&uc)[3])
{
  const int i = n % g.NX;
  const int j = (n / g.NX) % g.NY;
  const int k = n / (g.NX * g.NY);
  acc[0] = acc[1] = acc[2] = 0.0;
  double ul[2][9][3];
  double Ev[4];
  // elements below the node: node layers k-1 (bz = 0) and k (bz = 1)
  load_layer(u, g, i, j, k - 1, ul[0]);
  load_layer(u, g, i, j, k, ul[1]);
#pragma unroll
  for(int sy = 0; sy < 2; sy++)
#pragma unroll
    for(int sx = 0; sx < 2; sx++)
      Ev[sy * 2 + sx] = load_E(E, g, i - 1 + sx, j - 1 + sy, k - 1);
  layer_contrib<0>(ke, ul, Ev, acc);
  uc[0] = ul[1][4][0];
  uc[1] = ul[1][4][1];
  uc[2] = ul[1][4][2];
  // elements above: node layers k (bz = 0) and k+1 (bz = 1)
#pragma unroll
  for(int s = 0; s < 9; s++)
#pragma unroll
    for(int d = 0; d < 3; d++)
      ul[0][s][d] = ul[1][s][d];
  load_layer(u, g, i, j, k + 1, ul[1]);
#pragma unroll
  for(int sy = 0; sy < 2; sy++)
#pragma unroll
    for(int sx = 0; sx < 2; sx++)
      Ev[sy * 2 + sx] = load_E(E, g, i - 1 + sx, j - 1 + sy, k);
  layer_contrib<1>(ke, ul, Ev, acc);
}

} // namespace icarat_b200
