// Per-node stiffness stencil shared by the operator kernels (FP64 and FP32).
//
// (K u)_n = sum_{e containing n} E_e Ke0[rows of n in e] u_e, evaluated by
// node ownership: the thread of node n gathers the 27 nodal displacements
// around it and the moduli of its (up to) 8 elements, so no two threads
// write the same output and no atomics or colouring are needed.  Ke0 is a
// by-value kernel parameter (constant bank).
#pragma once
#include "internal.cuh"

namespace icarat_b200
{

// element matrix of the value type T (the FP32 copy is rounded from FP64)
template <typename T> struct KeOf;
template <> struct KeOf<double>
{
  using type = KeParam;
};
template <> struct KeOf<float>
{
  using type = KeParamF;
};

// local node number of the corner (lx, ly, lz) of a hexa8
// (mesh_icarat.hpp:489-509 order)
__host__ __device__ constexpr int local_node(int lx, int ly, int lz)
{
  return 4 * lz + (ly ? (lx ? 2 : 3) : (lx ? 1 : 0));
}

// One z-layer of 4 elements around node (i,j,k): SZ = 0 are the elements
// below the node (element k index k-1), SZ = 1 the ones above.  ul[l][s]
// holds the displacements of node layer k - 1 + SZ + l, s = (dy+1)*3+(dx+1).
//
// The box element is symmetric under reflection in its mid-planes, so its
// 3x3 blocks satisfy Ke0[a][b] = S_a K^_beta S_a with beta = |b - a| (per
// axis), K^_beta = Ke0[local node 0][local node beta] and S_a =
// diag((-1)^a_x, (-1)^a_y, (-1)^a_z).  The loop therefore runs over the 8
// canonical blocks: each block's 9 coefficients are read once and serve the 4
// elements of the layer (the signs are free FMA operand negations), and the
// 12 partial sums t[element][row] are independent accumulation chains.
template <int SZ, typename T, typename KP>
__device__ __forceinline__ void layer_contrib(const KP &ke, const T (&ul)[2][9][3],
                                              const T (&Ev)[4], T (&acc)[3])
{
  T t[4][3];
#pragma unroll
  for(int e = 0; e < 4; e++)
    t[e][0] = t[e][1] = t[e][2] = T(0);
#pragma unroll
  for(int bz = 0; bz < 2; bz++)
#pragma unroll
    for(int by = 0; by < 2; by++)
#pragma unroll
      for(int bx = 0; bx < 2; bx++)
      {
        const int lb = local_node(bx, by, bz);
        T kb[9];
#pragma unroll
        for(int c = 0; c < 3; c++)
#pragma unroll
          for(int d = 0; d < 3; d++)
            kb[3 * c + d] = ke.k[c * 24 + 3 * lb + d];
#pragma unroll
        for(int sy = 0; sy < 2; sy++)
#pragma unroll
          for(int sx = 0; sx < 2; sx++)
          {
            // element (sx, sy, SZ): the node's local corner a = 1 - s, the
            // neighbour at canonical offset beta is n + beta * (2 s - 1)
            const int ax = 1 - sx, ay = 1 - sy, az = 1 - SZ;
            const int dx = bx * (2 * sx - 1), dy = by * (2 * sy - 1);
            const int l = bz * (2 * SZ - 1) + 1 - SZ;
            const int s = (dy + 1) * 3 + (dx + 1);
            const int ac[3] = {ax, ay, az};
            const int e = sy * 2 + sx;
#pragma unroll
            for(int c = 0; c < 3; c++)
#pragma unroll
              for(int d = 0; d < 3; d++)
              {
                const bool neg = (c != d) && ((ac[c] + ac[d]) & 1);
                const T k = neg ? -kb[3 * c + d] : kb[3 * c + d];
                t[e][c] = fma(k, ul[l][s][d], t[e][c]);
              }
          }
      }
#pragma unroll
  for(int e = 0; e < 4; e++)
#pragma unroll
    for(int c = 0; c < 3; c++)
      acc[c] = fma(Ev[e], t[e][c], acc[c]);
}

// CG = true loads through L2 only (ld.global.cg): for vectors that the same
// (persistent) kernel rewrites between grid-wide barriers, where the
// read-only path could serve stale lines.
template <typename T, bool CG = false>
__device__ __forceinline__ void load_layer(const T *__restrict__ u, const GridDev &g,
                                           int i, int j, int kk, T (&L)[9][3])
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
        L[s][d] = in ? (CG ? __ldcg(u + (long)d * g.numnp + m) : __ldg(u + (long)d * g.numnp + m))
                     : T(0);
    }
}

template <typename T>
__device__ __forceinline__ T load_E(const T *__restrict__ E, const GridDev &g, int ei,
                                    int ej, int ek)
{
  const bool in = ei >= 0 && ei < g.nx && ej >= 0 && ej < g.ny && ek >= 0 &&
                  ek < g.nz;
  return in ? __ldg(E + ei + (long)ej * g.nx + (long)ek * g.nx * g.ny) : T(0);
}

// (K u) at node n (unmasked) and the node's own displacement uc.
template <typename T, typename KP, bool CG = false>
__device__ __forceinline__ void node_Ku(const GridDev &g, const KP &ke,
                                        const T *__restrict__ E,
                                        const T *__restrict__ u, int n, T (&acc)[3],
                                        T (&uc)[3])
{
  const int i = n % g.NX;
  const int j = (n / g.NX) % g.NY;
  const int k = n / (g.NX * g.NY);
  acc[0] = acc[1] = acc[2] = T(0);
  T ul[2][9][3];
  T Ev[4];
  // elements below the node: node layers k-1 (bz = 0) and k (bz = 1)
  load_layer<T, CG>(u, g, i, j, k - 1, ul[0]);
  load_layer<T, CG>(u, g, i, j, k, ul[1]);
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
  load_layer<T, CG>(u, g, i, j, k + 1, ul[1]);
#pragma unroll
  for(int sy = 0; sy < 2; sy++)
#pragma unroll
    for(int sx = 0; sx < 2; sx++)
      Ev[sy * 2 + sx] = load_E(E, g, i - 1 + sx, j - 1 + sy, k);
  layer_contrib<1>(ke, ul, Ev, acc);
}

} // namespace icarat_b200
