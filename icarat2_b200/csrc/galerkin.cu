// Galerkin coarse operators of the geometric multigrid (no reference
// counterpart: the reference has no multigrid).
//
// With trilinear prolongation on nested voxel grids every fine node inside a
// coarse cell is interpolated from that cell's 8 corners only, so the
// Galerkin product A_{l+1} = P^T A_l P is the assembly of per-cell 24x24
// matrices
//   Kc_C = sum over the 8 children s of C:  P_s^T M_s Kf_s M_s P_s,
// Kf_s the child's own matrix (level 0: E_e Ke0; level l >= 1: the child
// cell's Kc), M_s the child's constrained components (zeroed), P_s the
// child's 24 x 24 interpolation from C's corners (weights 1, 1/2, 0 per axis
// for a child node at fine coordinate 2 I, 2 I + 1, 2 I + 2).  Components of
// C's corners that the coarse level constrains are zeroed as well, so the
// assembled operator is D_c P^T D_f A D_f P D_c, the masked fine operator the
// rediscretised hierarchy approximates.
//
// Each coarse level stores its cell matrices (input of the next level) and
// the assembled node stencil, which the coarse levels' Chebyshev steps and
// residuals read (and the coarsest level's dense matrix).  The stencil is
// symmetric, so only the 14 neighbour blocks o >= 13 (o = 9 (dz + 1) +
// 3 (dy + 1) + (dx + 1); 13 is the node itself) are stored, coefficient-major
// (entry (o, c, d) of node n at (9 (o - 13) + 3 c + d) numnp + n); block o < 13
// of node n is the transpose of block 26 - o of its neighbour n + off(o).  The
// Chebyshev bound of a Galerkin level is max over its cells of
// lambda_max(diag(Kc)^-1 Kc) (by power iteration in each cell, times 1.02):
// with A = sum_C Kc_C and D = sum_C diag(Kc_C), x^T A x <= max_C lambda_C
// x^T D x, the same element bound the rediscretised levels use for Ke0.
#include <algorithm>

#include "stencil.cuh"

namespace icarat_b200
{

namespace
{
constexpr int kGalThreads = 128;

// corner coordinates of local node a (mesh_icarat.hpp:489-509 order)
__device__ __forceinline__ void corner_of(int a, int &x, int &y, int &z)
{
  const int q = a & 3;
  x = (q == 1 || q == 2) ? 1 : 0;
  y = (q >= 2) ? 1 : 0;
  z = a >> 2;
}

// weight of coarse corner coordinate i (0/1) at child node coordinate f
// (0, 1, 2 across the coarse cell)
__device__ __forceinline__ double w1(int f, int i)
{
  return f == 1 ? 0.5 : ((f == 0) == (i == 0) ? 1.0 : 0.0);
}
} // namespace

// Cell matrices of level 1 from E for the cells none of whose 27 child
// nodes has a constrained component (flag 0; then no corner has one either,
// a corner being a child node): Kc = sum_s E_s G_s, G_s = P_s^T Ke0 P_s
// (computed once on the host).  Thread per (cell, entry).  Their Chebyshev
// bound is max_s lambda_max(diag(G_s)^-1 G_s), a constant the host folds
// into the level's bound: x^T Kc x = sum_s E_s x^T G_s x <= max_s lambda_s
// x^T diag(Kc) x.
__global__ void k_gal_cells_free(GridDev f, GridDev c, const double *__restrict__ E,
                                 const double *__restrict__ G,
                                 const uint8_t *__restrict__ flag, double *__restrict__ Kc)
{
  const long total = 576L * c.nelx;
  for(long id = blockIdx.x * (long)blockDim.x + threadIdx.x; id < total;
      id += (long)gridDim.x * blockDim.x)
  {
    const int cell = (int)(id / 576), k = (int)(id % 576);
    if(flag[cell])
      continue;
    const int CI = cell % c.nx, CJ = (cell / c.nx) % c.ny, CK = cell / (c.nx * c.ny);
    double sum = 0.0;
#pragma unroll
    for(int q = 0; q < 8; q++)
    {
      const double e = E[(2 * CI + (q & 1)) + (2 * CJ + ((q >> 1) & 1)) * f.nx +
                         (2 * CK + (q >> 2)) * f.nx * f.ny];
      sum = fma(e, G[q * 576 + k], sum);
    }
    Kc[id] = sum;
  }
}

// Cell matrices of level l + 1 from level l, in general (block per coarse
// cell of `cells`, all cells when it is null): for each child q, its matrix
// with the rows and columns of constrained child components zeroed (M Kf M),
// T = Kf W_q, Kc += W_q^T T (W_q: the 8 x 8 node weights of P_q, per
// component); corner components the coarse level constrains are zeroed at
// the end.  Then the cell's bound lambda_max(diag(Kc)^-1 Kc) by power
// iteration (atomic max into *lmax, which starts at 0).
// Kf: level-l cell matrices (nullptr: level 0, E_e Ke0).
__global__ void __launch_bounds__(kGalThreads)
    k_gal_cells(GridDev f, GridDev c, KeParam ke, const double *__restrict__ E,
                const double *__restrict__ Kf, const uint8_t *__restrict__ fix_f,
                const uint8_t *__restrict__ fix_c, const int *__restrict__ cells, int ncells,
                double *__restrict__ Kc, double *__restrict__ lmax)
{
  __shared__ double sk[576];        // the child's matrix
  __shared__ double st[576];        // Kf W_q
  __shared__ double sc[576];        // this cell's matrix
  __shared__ double wt[8][8][8];    // wt[q][a][i]: weight of corner i at node a of child q
  __shared__ unsigned char mf[27];  // constrained bits of the 27 child nodes
  __shared__ unsigned char mc[8];   // constrained bits of the 8 corners
  __shared__ double v[24], y[24], dinv[24];
  __shared__ double lam;
  const int t = threadIdx.x;
  for(int idx = t; idx < 512; idx += blockDim.x)
  {
    const int q = idx >> 6, a = (idx >> 3) & 7, i = idx & 7;
    int ax, ay, az, ix, iy, iz;
    corner_of(a, ax, ay, az);
    corner_of(i, ix, iy, iz);
    wt[q][a][i] = w1((q & 1) + ax, ix) * w1(((q >> 1) & 1) + ay, iy) * w1((q >> 2) + az, iz);
  }
  for(int item = blockIdx.x; item < ncells; item += gridDim.x)
  {
    const int cell = cells ? cells[item] : item;
    const int CI = cell % c.nx, CJ = (cell / c.nx) % c.ny, CK = cell / (c.nx * c.ny);
    if(t < 27)
    {
      const int fx = t % 3, fy = (t / 3) % 3, fz = t / 9;
      mf[t] = fix_f[(2 * CI + fx) + (2 * CJ + fy) * f.NX + (2 * CK + fz) * f.NX * f.NY];
    }
    if(t < 8)
    {
      int x, y0, z;
      corner_of(t, x, y0, z);
      mc[t] = fix_c[(CI + x) + (CJ + y0) * c.NX + (CK + z) * c.NX * c.NY];
    }
    for(int k = t; k < 576; k += blockDim.x)
      sc[k] = 0.0;
    for(int q = 0; q < 8; q++)
    {
      __syncthreads(); // mf, sc ready; the previous child's st consumed
      const int sx = q & 1, sy = (q >> 1) & 1, sz = q >> 2;
      const int e = (2 * CI + sx) + (2 * CJ + sy) * f.nx + (2 * CK + sz) * f.nx * f.ny;
      for(int k = t; k < 576; k += blockDim.x)
      {
        const int r = k / 24, col = k % 24;
        const int ra = r / 3, rc = r % 3, ca = col / 3, cd = col % 3;
        int ax, ay, az, bx, by, bz;
        corner_of(ra, ax, ay, az);
        corner_of(ca, bx, by, bz);
        const bool fr = (mf[(sx + ax) + 3 * (sy + ay) + 9 * (sz + az)] >> rc) & 1u;
        const bool fc = (mf[(sx + bx) + 3 * (sy + by) + 9 * (sz + bz)] >> cd) & 1u;
        sk[k] = (fr || fc) ? 0.0 : (Kf ? Kf[(long)e * 576 + k] : E[e] * ke.k[k]);
      }
      __syncthreads();
      // st[(a, c)][(j, d)] = sum_b sk[(a, c)][(b, d)] w[q][b][j]
      for(int k = t; k < 576; k += blockDim.x)
      {
        const int r = k / 24, j = (k % 24) / 3, d = k % 3;
        double sum = 0.0;
#pragma unroll
        for(int b = 0; b < 8; b++)
          sum = fma(sk[r * 24 + 3 * b + d], wt[q][b][j], sum);
        st[k] = sum;
      }
      __syncthreads();
      // sc[(i, c)][col] += sum_a w[q][a][i] st[(a, c)][col]
      for(int k = t; k < 576; k += blockDim.x)
      {
        const int i = (k / 24) / 3, cc = (k / 24) % 3, col = k % 24;
        double sum = sc[k];
#pragma unroll
        for(int a = 0; a < 8; a++)
          sum = fma(wt[q][a][i], st[(3 * a + cc) * 24 + col], sum);
        sc[k] = sum;
      }
    }
    __syncthreads();
    // corner components the coarse level constrains; exact symmetry (the
    // mean of the two triangles) and the output
    for(int k = t; k < 576; k += blockDim.x)
    {
      const int r = k / 24, col = k % 24;
      const bool fx = ((mc[r / 3] >> (r % 3)) & 1u) || ((mc[col / 3] >> (col % 3)) & 1u);
      const double vsym = 0.5 * (sc[r * 24 + col] + sc[col * 24 + r]);
      Kc[(long)cell * 576 + k] = fx ? 0.0 : vsym;
      st[k] = fx ? 0.0 : vsym;
    }
    __syncthreads();
    // lambda_max(diag(Kc)^-1 Kc) over the cell's unconstrained components:
    // power iteration on D^-1/2 Kc D^-1/2 (one warp)
    if(t < 32)
    {
      if(t < 24)
      {
        const double dg = st[t * 24 + t];
        dinv[t] = dg > 0.0 ? 1.0 / sqrt(dg) : 0.0;
        v[t] = dinv[t] > 0.0 ? 1.0 + 0.01 * t : 0.0;
      }
      __syncwarp();
      double nrm = 0.0;
      for(int it = 0; it < 60; it++)
      {
        if(t < 24)
        {
          double sum = 0.0;
          for(int k = 0; k < 24; k++) // column t of the symmetric matrix: no bank conflicts
            sum = fma(st[k * 24 + t] * dinv[k], v[k], sum);
          y[t] = dinv[t] * sum;
        }
        __syncwarp();
        double q2 = t < 24 ? y[t] * y[t] : 0.0;
        for(int o = 16; o > 0; o >>= 1)
          q2 += __shfl_xor_sync(0xffffffffu, q2, o);
        nrm = sqrt(q2);
        if(t < 24)
          v[t] = nrm > 0.0 ? y[t] / nrm : 0.0;
        __syncwarp();
      }
      if(t == 0)
        lam = nrm;
    }
    __syncthreads();
    if(t == 0 && lam > 0.0)
      atomicMax(reinterpret_cast<unsigned long long *>(lmax),
                (unsigned long long)__double_as_longlong(1.02 * lam));
    __syncthreads();
  }
}

// Node stencil of a Galerkin level from its cell matrices (thread per node
// and neighbour offset), and the Jacobi inverse diagonal.
__global__ void k_gal_stencil(GridDev g, const double *__restrict__ Kc,
                              const uint8_t *__restrict__ fix, double *__restrict__ S,
                              double *__restrict__ invd)
{
  const long total = 14L * g.numnp;
  for(long id = blockIdx.x * (long)blockDim.x + threadIdx.x; id < total;
      id += (long)gridDim.x * blockDim.x)
  {
    const int n = (int)(id % g.numnp), o = 13 + (int)(id / g.numnp);
    const int X = n % g.NX, Y = (n / g.NX) % g.NY, Z = n / (g.NX * g.NY);
    const int ox = o % 3 - 1, oy = (o / 3) % 3 - 1, oz = o / 9 - 1;
    double blk[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    const int X2 = X + ox, Y2 = Y + oy, Z2 = Z + oz;
    if(X2 >= 0 && X2 < g.NX && Y2 >= 0 && Y2 < g.NY && Z2 >= 0 && Z2 < g.NZ)
    {
      // cells containing both nodes, in ascending cell order
      for(int cz = (Z > Z2 ? Z : Z2) - 1; cz <= (Z < Z2 ? Z : Z2); cz++)
        for(int cy = (Y > Y2 ? Y : Y2) - 1; cy <= (Y < Y2 ? Y : Y2); cy++)
          for(int cx = (X > X2 ? X : X2) - 1; cx <= (X < X2 ? X : X2); cx++)
          {
            if(cx < 0 || cy < 0 || cz < 0 || cx >= g.nx || cy >= g.ny || cz >= g.nz)
              continue;
            const int la = local_node(X - cx, Y - cy, Z - cz);
            const int lb = local_node(X2 - cx, Y2 - cy, Z2 - cz);
            const double *K = Kc + ((long)cx + (long)cy * g.nx + (long)cz * g.nx * g.ny) * 576;
#pragma unroll
            for(int c = 0; c < 3; c++)
#pragma unroll
              for(int d = 0; d < 3; d++)
                blk[3 * c + d] += K[(3 * la + c) * 24 + 3 * lb + d];
          }
    }
#pragma unroll
    for(int k = 0; k < 9; k++)
      S[(9L * (o - 13) + k) * g.numnp + n] = blk[k];
    if(o == 13)
    {
      const unsigned fx = fix[n];
#pragma unroll
      for(int c = 0; c < 3; c++)
        invd[(long)c * g.numnp + n] =
            (((fx >> c) & 1u) || blk[4 * c] <= 0.0) ? 0.0 : 1.0 / blk[4 * c];
    }
  }
}

// Chebyshev coefficients of every Galerkin level from its bound: per level
// kGalCoef entries, [0] = 1 / theta, then (c1, c2) of steps 1, 2, ...  (the
// sequence of smooth() in multigrid.cu on [0.1 lmax, lmax])
__global__ void k_gal_coefs(int levels, const double *__restrict__ lmax, double lam1,
                            double *__restrict__ coef)
{
  const int l = threadIdx.x;
  if(l >= levels)
    return;
  // level 1: the cells of the fast form contribute the constant bound lam1
  const double lb = l == 1 ? fmax(lmax[l], lam1) : lmax[l];
  const double lm = lb > 0.0 ? lb : 1.0;
  const double lo = 0.1 * lm;
  const double theta = 0.5 * (lm + lo), delta = 0.5 * (lm - lo);
  const double sigma = theta / delta;
  double rho_old = 1.0 / sigma;
  double *cf = coef + (long)l * kGalCoef;
  cf[0] = 1.0 / theta;
  for(int k = 1; 2 * k < kGalCoef; k++)
  {
    const double rho = 1.0 / (2.0 * sigma - rho_old);
    cf[2 * k - 1] = rho * rho_old;
    cf[2 * k] = 2.0 * rho / delta;
    rho_old = rho;
  }
}

// Stencil products, 9 threads per node: block (32, 9), threadIdx.x the node
// of the block's 32, threadIdx.y = 3 c + p the row component c and the
// neighbour slab dz = p - 1 (9 neighbours x 3 components each).  The three
// slab sums of a row are added in slab order by the p = 0 thread.  Short
// dependent chains and many threads per node keep the small coarse levels
// from waiting on one long chain of loads per node.
constexpr int kStNodes = 32;

// A[(n, c), (m, d)] of neighbour block o (m = n + off(o)) from the half
// storage
template <typename T>
__device__ __forceinline__ T st_coef(const T *__restrict__ S, int numnp, long n, long m, int o,
                                     int c, int d)
{
  return o >= 13 ? S[(9L * (o - 13) + 3 * c + d) * numnp + n]
                 : S[(9L * (13 - o) + 3 * d + c) * numnp + m];
}

template <int DZ, typename T>
__device__ __forceinline__ T stencil_slab(const GridDev &g, const T *__restrict__ S,
                                          const T *__restrict__ x, int n, int c)
{
  const int X = n % g.NX, Y = (n / g.NX) % g.NY, Z = n / (g.NX * g.NY);
  const bool zin = Z + DZ >= 0 && Z + DZ < g.NZ;
  // every load is issued (out-of-mesh neighbours read node n and count 0),
  // so that the 54 loads of a slab need not wait for one another
  T acc = T(0);
#pragma unroll
  for(int dy = -1; dy <= 1; dy++)
#pragma unroll
    for(int dx = -1; dx <= 1; dx++)
    {
      const bool in =
          zin && X + dx >= 0 && X + dx < g.NX && Y + dy >= 0 && Y + dy < g.NY;
      constexpr int o0 = 9 * (DZ + 1);
      const int o = o0 + 3 * (dy + 1) + (dx + 1);
      const long m = in ? n + dx + (long)dy * g.NX + (long)DZ * g.NX * g.NY : n;
#pragma unroll
      for(int d = 0; d < 3; d++)
      {
        const T a = st_coef(S, g.numnp, n, m, o, c, d);
        acc = fma(in ? a : T(0), x[(long)d * g.numnp + m], acc);
      }
    }
  return acc;
}

template <typename T>
__device__ __forceinline__ T stencil_slab_any(const GridDev &g, const T *__restrict__ S,
                                              const T *__restrict__ x, int n, int c, int p)
{
  // p is uniform over a warp (threadIdx.y)
  return p == 0 ? stencil_slab<-1>(g, S, x, n, c)
                : (p == 1 ? stencil_slab<0>(g, S, x, n, c) : stencil_slab<1>(g, S, x, n, c));
}

// (A x)_{n, c} for the block's node lane; true on the thread that holds the
// row sum (p = 0) of a node inside the level.  Every thread of the block
// calls it (it synchronises the block).
template <typename T>
__device__ __forceinline__ bool stencil_row(const GridDev &g, const T *__restrict__ S,
                                            const T *__restrict__ x, int n, double (&ps)[9][kStNodes],
                                            T &row)
{
  const int c = threadIdx.y / 3, p = threadIdx.y % 3;
  ps[threadIdx.y][threadIdx.x] = n < g.numnp ? (double)stencil_slab_any(g, S, x, n, c, p) : 0.0;
  __syncthreads();
  row = T((ps[3 * c][threadIdx.x] + ps[3 * c + 1][threadIdx.x]) + ps[3 * c + 2][threadIdx.x]);
  const bool mine = p == 0 && n < g.numnp;
  __syncthreads();
  return mine;
}

// first Chebyshev step from x = 0: d = invd b / theta, x = d
template <typename T>
__global__ void k_st_first(int n, const T *__restrict__ b, const T *__restrict__ invd,
                           const double *__restrict__ coef, T *__restrict__ x,
                           T *__restrict__ d, const int *__restrict__ halt)
{
  chain_wait();
  if(halted(halt))
    return;
  const T it = T(coef[0]);
  for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
  {
    const T di = invd[i] * b[i] * it;
    d[i] = di;
    x[i] = di;
  }
}

// Chebyshev step k of a stencil level: d = c1 d + c2 invd (b - A x), xo = x + d
// (k = 0: c1 = 0, c2 = 1 / theta); block (kStNodes, 9)
template <typename T>
__global__ void __launch_bounds__(kStNodes * 9, 3)
    k_st_cheb(GridDev g, const T *__restrict__ S, const uint8_t *__restrict__ fix,
              const T *__restrict__ invd, const T *__restrict__ b, const T *__restrict__ x,
              T *__restrict__ d, T *__restrict__ xo, const double *__restrict__ coef, int k,
              const int *__restrict__ halt)
{
  chain_wait();
  if(halted(halt))
    return;
  __shared__ double ps[9][kStNodes];
  const T c1 = k == 0 ? T(0) : T(coef[2 * k - 1]);
  const T c2 = k == 0 ? T(coef[0]) : T(coef[2 * k]);
  const int q = threadIdx.y / 3;
  for(int nb = blockIdx.x * kStNodes; nb < g.numnp; nb += gridDim.x * kStNodes)
  {
    const int n = nb + threadIdx.x;
    T acc;
    if(!stencil_row(g, S, x, n, ps, acc))
      continue;
    const long id = (long)q * g.numnp + n;
    T dn = 0;
    if(!((fix[n] >> q) & 1u))
      dn = (c1 != T(0) ? c1 * d[id] : T(0)) + c2 * invd[id] * (b[id] - acc);
    d[id] = dn;
    xo[id] = x[id] + dn;
  }
}

// r = b - A x (constrained rows 0); block (kStNodes, 9)
template <typename T>
__global__ void __launch_bounds__(kStNodes * 9, 3)
    k_st_residual(GridDev g, const T *__restrict__ S, const uint8_t *__restrict__ fix,
                  const T *__restrict__ b, const T *__restrict__ x, T *__restrict__ r,
                  const int *__restrict__ halt)
{
  chain_wait();
  if(halted(halt))
    return;
  __shared__ double ps[9][kStNodes];
  const int q = threadIdx.y / 3;
  for(int nb = blockIdx.x * kStNodes; nb < g.numnp; nb += gridDim.x * kStNodes)
  {
    const int n = nb + threadIdx.x;
    T acc;
    if(!stencil_row(g, S, x, n, ps, acc))
      continue;
    const long id = (long)q * g.numnp + n;
    r[id] = ((fix[n] >> q) & 1u) ? T(0) : b[id] - acc;
  }
}

// launch shape of k_st_cheb / k_st_residual
dim3 st_block()
{
  return dim3(kStNodes, 9);
}
int st_blocks(int numnp)
{
  return (numnp + kStNodes - 1) / kStNodes;
}

// dense coarsest matrix from the coarsest level's stencil (thread per free
// row; entries of constrained columns are skipped)
__global__ void k_coarse_assemble_st(GridDev g, const double *__restrict__ S,
                                     const int *__restrict__ rowmap,
                                     const int *__restrict__ colmap, int nfree,
                                     double *__restrict__ A)
{
  for(int r = blockIdx.x * blockDim.x + threadIdx.x; r < nfree; r += gridDim.x * blockDim.x)
  {
    const int full = rowmap[r];
    const int c = full / g.numnp, n = full % g.numnp;
    const int X = n % g.NX, Y = (n / g.NX) % g.NY, Z = n / (g.NX * g.NY);
    double *row = A + (long)r * nfree;
    for(int o = 0; o < 27; o++)
    {
      const int ox = o % 3 - 1, oy = (o / 3) % 3 - 1, oz = o / 9 - 1;
      const int X2 = X + ox, Y2 = Y + oy, Z2 = Z + oz;
      if(X2 < 0 || X2 >= g.NX || Y2 < 0 || Y2 >= g.NY || Z2 < 0 || Z2 >= g.NZ)
        continue;
      const int m = X2 + Y2 * g.NX + Z2 * g.NX * g.NY;
      for(int d = 0; d < 3; d++)
      {
        const int col = colmap[3L * m + d];
        if(col >= 0)
          row[col] = st_coef(S, g.numnp, n, m, o, c, d);
      }
    }
  }
}

// The 8 child matrices G_s = P_s^T Ke0 P_s (row-major 24 x 24, the order of
// k_gal_cells) and max_s lambda_max(diag(G_s)^-1 G_s), on the host.
double galerkin_child_matrices(const double *ke0, double *G)
{
  auto corner = [](int a, int &x, int &y, int &z)
  {
    const int q = a & 3;
    x = (q == 1 || q == 2) ? 1 : 0;
    y = q >= 2 ? 1 : 0;
    z = a >> 2;
  };
  auto w = [](int f, int i) { return f == 1 ? 0.5 : ((f == 0) == (i == 0) ? 1.0 : 0.0); };
  double lam = 0.0;
  for(int s = 0; s < 8; s++)
  {
    const int sx = s & 1, sy = (s >> 1) & 1, sz = s >> 2;
    double P[8][8]; // P[a][i]: weight of corner i at child node a
    for(int a = 0; a < 8; a++)
      for(int i = 0; i < 8; i++)
      {
        int ax, ay, az, ix, iy, iz;
        corner(a, ax, ay, az);
        corner(i, ix, iy, iz);
        P[a][i] = w(sx + ax, ix) * w(sy + ay, iy) * w(sz + az, iz);
      }
    double *g = G + 576 * s;
    for(int row = 0; row < 24; row++)
      for(int col = 0; col < 24; col++)
      {
        const int i = row / 3, c = row % 3, j = col / 3, d = col % 3;
        double sum = 0.0;
        for(int a = 0; a < 8; a++)
        {
          if(P[a][i] == 0.0)
            continue;
          double inner = 0.0;
          for(int b = 0; b < 8; b++)
            if(P[b][j] != 0.0)
              inner += P[b][j] * ke0[(3 * a + c) * 24 + 3 * b + d];
          sum += P[a][i] * inner;
        }
        g[row * 24 + col] = sum;
      }
    for(int row = 0; row < 24; row++) // exact symmetry
      for(int col = 0; col < row; col++)
        g[col * 24 + row] = g[row * 24 + col];
    lam = std::max(lam, jacobi_bound(g));
  }
  return lam;
}

// host launches of the stencil-level kernels (the kernels stay in this
// translation unit); halt: the V-cycle stop flag (null: never stop)
template <typename T>
void st_first_launch(cudaStream_t st, int n, const T *b, const T *invd, const double *coef,
                     T *x, T *d, const int *halt)
{
  note_launch();
  launch_chained(k_st_first<T>, (n + 255) / 256, 256, 0, st, n, b, invd, coef, x, d, halt);
}
template <typename T>
void st_cheb_launch(cudaStream_t st, const GridDev &g, const T *S, const uint8_t *fix,
                    const T *invd, const T *b, const T *x, T *d, T *xo, const double *coef, int k,
                    const int *halt)
{
  note_launch();
  launch_chained(k_st_cheb<T>, st_blocks(g.numnp), st_block(), 0, st, g, S, fix, invd, b, x, d,
                 xo, coef, k, halt);
}
template <typename T>
void st_residual_launch(cudaStream_t st, const GridDev &g, const T *S, const uint8_t *fix,
                        const T *b, const T *x, T *r, const int *halt)
{
  note_launch();
  launch_chained(k_st_residual<T>, st_blocks(g.numnp), st_block(), 0, st, g, S, fix, b, x, r,
                 halt);
}
template void st_first_launch<double>(cudaStream_t, int, const double *, const double *,
                                      const double *, double *, double *, const int *);
template void st_first_launch<float>(cudaStream_t, int, const float *, const float *,
                                     const double *, float *, float *, const int *);
template void st_cheb_launch<double>(cudaStream_t, const GridDev &, const double *,
                                     const uint8_t *, const double *, const double *,
                                     const double *, double *, double *, const double *, int,
                                     const int *);
template void st_cheb_launch<float>(cudaStream_t, const GridDev &, const float *,
                                    const uint8_t *, const float *, const float *, const float *,
                                    float *, float *, const double *, int, const int *);
template void st_residual_launch<double>(cudaStream_t, const GridDev &, const double *,
                                         const uint8_t *, const double *, const double *,
                                         double *, const int *);
template void st_residual_launch<float>(cudaStream_t, const GridDev &, const float *,
                                        const uint8_t *, const float *, const float *, float *,
                                        const int *);

} // namespace icarat_b200
