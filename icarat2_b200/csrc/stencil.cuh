// Per-node stiffness stencil shared by the operator kernels (FP64 and FP32).
//
// (K u)_n = sum_{e containing n} E_e Ke0[rows of n in e] u_e, evaluated by
// node ownership: the thread of node n gathers the 27 nodal displacements
// around it and the moduli of its (up to) 8 elements, so no two threads
// write the same output and no atomics or colouring are needed.  Ke0 is a
// by-value kernel parameter (constant bank).
#pragma once
#include <map>
#include <mutex>
#include <utility>

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

// Grid transfers of the geometric multigrid for one node (CG = true: loads
// through L2 only, for vectors rewritten inside a persistent launch).
// Restriction R = P^T: the 27 fine nodes around coarse node n with weights
// 1/2 per offset axis; s = (R r)_n before masking.
template <typename T, bool CG>
__device__ __forceinline__ void restrict_node(const GridDev &f, const GridDev &c,
                                              const T *__restrict__ rf, int n, T (&s)[3])
{
  const int I = n % c.NX, J = (n / c.NX) % c.NY, K = n / (c.NX * c.NY);
  s[0] = s[1] = s[2] = T(0);
#pragma unroll
  for(int dz = -1; dz <= 1; dz++)
#pragma unroll
    for(int dy = -1; dy <= 1; dy++)
#pragma unroll
      for(int dx = -1; dx <= 1; dx++)
      {
        const int i = 2 * I + dx, j = 2 * J + dy, k = 2 * K + dz;
        if(i < 0 || i >= f.NX || j < 0 || j >= f.NY || k < 0 || k >= f.NZ)
          continue;
        const T w = T((dx ? 0.5 : 1.0) * (dy ? 0.5 : 1.0) * (dz ? 0.5 : 1.0));
        const long m = i + (long)j * f.NX + (long)k * f.NX * f.NY;
#pragma unroll
        for(int q = 0; q < 3; q++)
          s[q] += w * (CG ? __ldcg(rf + (long)q * f.numnp + m) : rf[(long)q * f.numnp + m]);
      }
}

// Trilinear prolongation: s = (P xc) at fine node n (odd coordinates take
// both coarse neighbours with 1/2, even ones the coincident coarse node).
template <typename T, bool CG>
__device__ __forceinline__ void prolong_node(const GridDev &f, const GridDev &c,
                                             const T *__restrict__ xc, int n, T (&s)[3])
{
  const int i = n % f.NX, j = (n / f.NX) % f.NY, k = n / (f.NX * f.NY);
  const int I0 = i >> 1, J0 = j >> 1, K0 = k >> 1;
  const int I1 = I0 + (i & 1), J1 = J0 + (j & 1), K1 = K0 + (k & 1);
  const T wx = (i & 1) ? T(0.5) : T(1), wy = (j & 1) ? T(0.5) : T(1),
          wz = (k & 1) ? T(0.5) : T(1);
  s[0] = s[1] = s[2] = T(0);
#pragma unroll
  for(int cz = 0; cz < 2; cz++)
#pragma unroll
    for(int cy = 0; cy < 2; cy++)
#pragma unroll
      for(int cx = 0; cx < 2; cx++)
      {
        if((cx && !(i & 1)) || (cy && !(j & 1)) || (cz && !(k & 1)))
          continue;
        const int I = cx ? I1 : I0, J = cy ? J1 : J0, K = cz ? K1 : K0;
        const long m = I + (long)J * c.NX + (long)K * c.NX * c.NY;
        const T w = wx * wy * wz;
#pragma unroll
        for(int q = 0; q < 3; q++)
          s[q] += w * (CG ? __ldcg(xc + (long)q * c.numnp + m) : xc[(long)q * c.numnp + m]);
      }
}

// Column march.  The thread of node column (i, j) evaluates K u at the nodes
// (i, j, k), k0 <= k < k1, sweeping the element layers e = k0 - 1 .. k1 - 1
// once: element layer e closes node e (its elements above, SZ = 1) and opens
// node e + 1 (its elements below, SZ = 0), so every node layer's 27
// displacements and every element layer's 4 moduli are loaded once per
// column instead of once per node, and the x / y bounds tests are per column.
// The sums run in the order of node_Ku (below, then above), so the results
// are identical.  emit(k, acc, uc) receives each node's K u and its own
// displacement.
template <typename T, typename KP, bool CG = false, typename F>
__device__ __forceinline__ void column_Ku(const GridDev &g, const KP &ke,
                                          const T *__restrict__ E, const T *__restrict__ u,
                                          int i, int j, int k0, int k1, F &&emit)
{
  T ul[2][9][3];
  T below[3] = {T(0), T(0), T(0)};
  load_layer<T, CG>(u, g, i, j, k0 - 1, ul[0]);
  for(int e = k0 - 1; e < k1; e++)
  {
    load_layer<T, CG>(u, g, i, j, e + 1, ul[1]);
    T Ev[4];
#pragma unroll
    for(int sy = 0; sy < 2; sy++)
#pragma unroll
      for(int sx = 0; sx < 2; sx++)
        Ev[sy * 2 + sx] = load_E(E, g, i - 1 + sx, j - 1 + sy, e);
    if(e >= k0)
    {
      T acc[3] = {below[0], below[1], below[2]};
      layer_contrib<1>(ke, ul, Ev, acc);
      const T uc[3] = {ul[0][4][0], ul[0][4][1], ul[0][4][2]};
      emit(e, acc, uc);
    }
    if(e + 1 < k1)
    {
      below[0] = below[1] = below[2] = T(0);
      layer_contrib<0>(ke, ul, Ev, below);
    }
#pragma unroll
    for(int s = 0; s < 9; s++)
#pragma unroll
      for(int d = 0; d < 3; d++)
        ul[0][s][d] = ul[1][s][d];
  }
}

// Work items of a column march: ncol columns (NX NY rounded up to whole
// warps, so a warp never straddles two z chunks) times ceil(NZ / kc) chunks.
struct MarchPlan
{
  int kc, ncol;
  long items;
};

// node layers per chunk: the largest count that still gives every resident
// thread slot (slots) about two items, down to one layer per item on the
// small multigrid levels, which are latency-bound (their operands sit in L2,
// so the layers a short chunk re-reads cost little; results do not depend on
// the chunking)
inline MarchPlan march_plan(const GridDev &g, long slots)
{
  MarchPlan m;
  m.ncol = ((g.NX * g.NY + 31) / 32) * 32;
  int kc = g.NZ;
  while(kc > 1 && (long)m.ncol * ((g.NZ + kc - 1) / kc) < 2 * slots)
    kc = (kc + 1) / 2;
  m.kc = kc < 1 ? 1 : kc;
  m.items = (long)m.ncol * ((g.NZ + m.kc - 1) / m.kc);
  return m;
}

// resident threads of `kernel` at `threads` per block on the whole GPU
// (occupancy cached per kernel)
inline long resident_threads(const void *kernel, int threads, int sms)
{
  static std::mutex mu;
  static std::map<std::pair<const void *, int>, int> cache;
  std::lock_guard<std::mutex> lock(mu);
  auto key = std::make_pair(kernel, threads);
  auto it = cache.find(key);
  int occ;
  if(it == cache.end())
  {
    occ = 0;
    if(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kernel, threads, 0) != cudaSuccess ||
       occ < 1)
      occ = 1;
    cache[key] = occ;
  }
  else
    occ = it->second;
  return (long)occ * threads * sms;
}

// plan and block count of a column-march launch of `kernel`
inline MarchPlan march_launch(const GridDev &g, const void *kernel, int threads, int sms,
                              int &blocks)
{
  const MarchPlan m = march_plan(g, resident_threads(kernel, threads, sms));
  const long b = (m.items + threads - 1) / threads;
  blocks = (int)(b < 1 ? 1 : b);
  return m;
}

// the column and z range of item t; false for the padding columns
__device__ __forceinline__ bool march_item(const GridDev &g, const MarchPlan &m, long t,
                                           int &i, int &j, int &k0, int &k1)
{
  const int col = (int)(t % m.ncol);
  const int chunk = (int)(t / m.ncol);
  if(col >= g.NX * g.NY)
    return false;
  i = col % g.NX;
  j = col / g.NX;
  k0 = chunk * m.kc;
  k1 = k0 + m.kc < g.NZ ? k0 + m.kc : g.NZ;
  return true;
}

} // namespace icarat_b200
