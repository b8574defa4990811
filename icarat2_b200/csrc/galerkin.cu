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
// the assembled node stencil: per node 27 neighbour blocks of 3 x 3,
// coefficient-major (entry (o, c, d) of node n at (9 o + 3 c + d) numnp + n,
// o = 9 (dz + 1) + 3 (dy + 1) + (dx + 1)), which the coarse levels' Chebyshev
// steps and residuals read (and the coarsest level's dense matrix).  The
// Chebyshev bound of a Galerkin level is max over its cells of
// lambda_max(diag(Kc)^-1 Kc) (by power iteration in each cell, times 1.02):
// with A = sum_C Kc_C and D = sum_C diag(Kc_C), x^T A x <= max_C lambda_C
// x^T D x, the same element bound the rediscretised levels use for Ke0.
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

// Cell matrices of level l + 1 from level l (block per coarse cell), and the
// level's Chebyshev bound (atomic max into *lmax, which starts at 0).
// Kf: level-l cell matrices (nullptr: level 0, E_e Ke0).
__global__ void __launch_bounds__(kGalThreads)
    k_gal_cells(GridDev f, GridDev c, KeParam ke, const double *__restrict__ E,
                const double *__restrict__ Kf, const uint8_t *__restrict__ fix_f,
                const uint8_t *__restrict__ fix_c, double *__restrict__ Kc,
                double *__restrict__ lmax)
{
  __shared__ double sk[8][576]; // the children's matrices
  __shared__ double sc[576];     // this cell's matrix
  __shared__ unsigned char mf[27]; // constrained bits of the 27 child nodes
  __shared__ unsigned char mc[8];  // constrained bits of the 8 corners
  __shared__ double v[24], y[24], dinv[24];
  __shared__ double lam;
  const int t = threadIdx.x;
  const int cell = blockIdx.x;
  const int CI = cell % c.nx, CJ = (cell / c.nx) % c.ny, CK = cell / (c.nx * c.ny);
  // children s = sx + 2 sy + 4 sz: fine element (2 CI + sx, 2 CJ + sy, 2 CK + sz)
  for(int idx = t; idx < 8 * 576; idx += blockDim.x)
  {
    const int s = idx / 576, k = idx % 576;
    const int e = (2 * CI + (s & 1)) + (2 * CJ + ((s >> 1) & 1)) * f.nx +
                  (2 * CK + (s >> 2)) * f.nx * f.ny;
    sk[s][k] = Kf ? Kf[(long)e * 576 + k] : E[e] * ke.k[k];
  }
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
  __syncthreads();
  // the lower triangle (row >= col), mirrored: the cell matrix is exactly
  // symmetric
  for(int ent = t; ent < 300; ent += blockDim.x)
  {
    int row = 0;
    while((row + 1) * (row + 2) / 2 <= ent)
      row++;
    const int col = ent - row * (row + 1) / 2;
    const int i = row / 3, cc = row % 3, j = col / 3, dd = col % 3;
    double sum = 0.0;
    if(!((mc[i] >> cc) & 1u) && !((mc[j] >> dd) & 1u))
    {
      int ix, iy, iz, jx, jy, jz;
      corner_of(i, ix, iy, iz);
      corner_of(j, jx, jy, jz);
      for(int s = 0; s < 8; s++)
      {
        const int sx = s & 1, sy = (s >> 1) & 1, sz = s >> 2;
        for(int a = 0; a < 8; a++)
        {
          int ax, ay, az;
          corner_of(a, ax, ay, az);
          const int fa = (sx + ax) + 3 * (sy + ay) + 9 * (sz + az);
          const double wa = w1(sx + ax, ix) * w1(sy + ay, iy) * w1(sz + az, iz);
          if(wa == 0.0 || ((mf[fa] >> cc) & 1u))
            continue;
          double inner = 0.0;
          for(int b = 0; b < 8; b++)
          {
            int bx, by, bz;
            corner_of(b, bx, by, bz);
            const int fb = (sx + bx) + 3 * (sy + by) + 9 * (sz + bz);
            const double wb = w1(sx + bx, jx) * w1(sy + by, jy) * w1(sz + bz, jz);
            if(wb == 0.0 || ((mf[fb] >> dd) & 1u))
              continue;
            inner = fma(wb, sk[s][(3 * a + cc) * 24 + 3 * b + dd], inner);
          }
          sum = fma(wa, inner, sum);
        }
      }
    }
    sc[row * 24 + col] = sum;
    sc[col * 24 + row] = sum;
    Kc[(long)cell * 576 + row * 24 + col] = sum;
    Kc[(long)cell * 576 + col * 24 + row] = sum;
  }
  __syncthreads();
  // lambda_max(diag(Kc)^-1 Kc) over the cell's unconstrained components: power
  // iteration on D^-1/2 Kc D^-1/2 (one warp)
  if(t < 32)
  {
    if(t < 24)
    {
      const double dg = sc[t * 24 + t];
      dinv[t] = dg > 0.0 ? 1.0 / sqrt(dg) : 0.0;
      v[t] = dinv[t] > 0.0 ? 1.0 + 0.01 * t : 0.0;
    }
    __syncwarp();
    double nrm = 0.0;
    for(int it = 0; it < 60; it++)
    {
      if(t < 24)
      {
        double s = 0.0;
        for(int k = 0; k < 24; k++)
          s = fma(sc[t * 24 + k] * dinv[k], v[k], s);
        y[t] = dinv[t] * s;
      }
      __syncwarp();
      double q = t < 24 ? y[t] * y[t] : 0.0;
      for(int o = 16; o > 0; o >>= 1)
        q += __shfl_xor_sync(0xffffffffu, q, o);
      nrm = sqrt(q);
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
}

// Node stencil of a Galerkin level from its cell matrices (thread per node
// and neighbour offset), and the Jacobi inverse diagonal.
__global__ void k_gal_stencil(GridDev g, const double *__restrict__ Kc,
                              const uint8_t *__restrict__ fix, double *__restrict__ S,
                              double *__restrict__ invd)
{
  const long total = 27L * g.numnp;
  for(long id = blockIdx.x * (long)blockDim.x + threadIdx.x; id < total;
      id += (long)gridDim.x * blockDim.x)
  {
    const int n = (int)(id % g.numnp), o = (int)(id / g.numnp);
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
      S[(9L * o + k) * g.numnp + n] = blk[k];
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
__global__ void k_gal_coefs(int levels, const double *__restrict__ lmax,
                            double *__restrict__ coef)
{
  const int l = threadIdx.x;
  if(l >= levels)
    return;
  const double lm = lmax[l] > 0.0 ? lmax[l] : 1.0;
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

// (A x) at node n of a stencil level (unmasked)
template <typename T>
__device__ __forceinline__ void stencil_Ax(const GridDev &g, const T *__restrict__ S,
                                           const T *__restrict__ x, int n, T (&acc)[3])
{
  const int X = n % g.NX, Y = (n / g.NX) % g.NY, Z = n / (g.NX * g.NY);
  acc[0] = acc[1] = acc[2] = T(0);
#pragma unroll
  for(int o = 0; o < 27; o++)
  {
    const int ox = o % 3 - 1, oy = (o / 3) % 3 - 1, oz = o / 9 - 1;
    const int X2 = X + ox, Y2 = Y + oy, Z2 = Z + oz;
    if(X2 < 0 || X2 >= g.NX || Y2 < 0 || Y2 >= g.NY || Z2 < 0 || Z2 >= g.NZ)
      continue;
    const long m = n + ox + (long)oy * g.NX + (long)oz * g.NX * g.NY;
    const T u[3] = {x[m], x[(long)g.numnp + m], x[2L * g.numnp + m]};
#pragma unroll
    for(int c = 0; c < 3; c++)
#pragma unroll
      for(int d = 0; d < 3; d++)
        acc[c] = fma(S[(9L * o + 3 * c + d) * g.numnp + n], u[d], acc[c]);
  }
}

// first Chebyshev step from x = 0: d = invd b / theta, x = d
template <typename T>
__global__ void k_st_first(int n, const T *__restrict__ b, const T *__restrict__ invd,
                           const double *__restrict__ coef, T *__restrict__ x,
                           T *__restrict__ d)
{
  const T it = T(coef[0]);
  for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
  {
    const T di = invd[i] * b[i] * it;
    d[i] = di;
    x[i] = di;
  }
}

// Chebyshev step k of a stencil level: d = c1 d + c2 invd (b - A x), xo = x + d
// (k = 0: c1 = 0, c2 = 1 / theta)
template <typename T>
__global__ void k_st_cheb(GridDev g, const T *__restrict__ S, const uint8_t *__restrict__ fix,
                          const T *__restrict__ invd, const T *__restrict__ b,
                          const T *__restrict__ x, T *__restrict__ d, T *__restrict__ xo,
                          const double *__restrict__ coef, int k)
{
  const T c1 = k == 0 ? T(0) : T(coef[2 * k - 1]);
  const T c2 = k == 0 ? T(coef[0]) : T(coef[2 * k]);
  for(int n = blockIdx.x * blockDim.x + threadIdx.x; n < g.numnp; n += gridDim.x * blockDim.x)
  {
    T acc[3];
    stencil_Ax(g, S, x, n, acc);
    const unsigned f = fix[n];
#pragma unroll
    for(int q = 0; q < 3; q++)
    {
      const long id = (long)q * g.numnp + n;
      T dn = 0;
      if(!((f >> q) & 1u))
        dn = (c1 != T(0) ? c1 * d[id] : T(0)) + c2 * invd[id] * (b[id] - acc[q]);
      d[id] = dn;
      xo[id] = x[id] + dn;
    }
  }
}

// r = b - A x (constrained rows 0)
template <typename T>
__global__ void k_st_residual(GridDev g, const T *__restrict__ S,
                              const uint8_t *__restrict__ fix, const T *__restrict__ b,
                              const T *__restrict__ x, T *__restrict__ r)
{
  for(int n = blockIdx.x * blockDim.x + threadIdx.x; n < g.numnp; n += gridDim.x * blockDim.x)
  {
    T acc[3];
    stencil_Ax(g, S, x, n, acc);
    const unsigned f = fix[n];
#pragma unroll
    for(int q = 0; q < 3; q++)
      r[(long)q * g.numnp + n] = ((f >> q) & 1u) ? T(0) : b[(long)q * g.numnp + n] - acc[q];
  }
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
          row[col] = S[(9L * o + 3 * c + d) * g.numnp + n];
      }
    }
  }
}

template __global__ void k_st_first<double>(int, const double *, const double *,
                                            const double *, double *, double *);
template __global__ void k_st_first<float>(int, const float *, const float *, const double *,
                                           float *, float *);
template __global__ void k_st_cheb<double>(GridDev, const double *, const uint8_t *,
                                           const double *, const double *, const double *,
                                           double *, double *, const double *, int);
template __global__ void k_st_cheb<float>(GridDev, const float *, const uint8_t *,
                                          const float *, const float *, const float *, float *,
                                          float *, const double *, int);
template __global__ void k_st_residual<double>(GridDev, const double *, const uint8_t *,
                                               const double *, const double *, double *);
template __global__ void k_st_residual<float>(GridDev, const float *, const uint8_t *,
                                              const float *, const float *, float *);

} // namespace icarat_b200
