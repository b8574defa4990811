// Geometric multigrid preconditioner for the SIMP stiffness (no reference
// counterpart: the reference solves with Jacobi-PCG or a direct solver).
//
// Level l + 1 halves every axis of level l.  Coarse operators are
// rediscretised: a coarse element's modulus is the mean of its 8 children
// times 2 (a hexa8 stiffness scales with its edge length), so every level
// reuses the fine Ke0 and the matrix-free node stencil.  A coarse node is
// constrained where its coincident fine node is.  Transfers are trilinear
// prolongation P and restriction R = P^T.  Smoothing is a Chebyshev
// polynomial in D^-1 K on [0.1 lmax, lmax], where lmax is the element bound
// of the Jacobi-scaled Ke0 (a rigorous bound for every SIMP design), applied
// identically before and after the coarse correction so that the V-cycle is
// a symmetric positive definite preconditioner.  The coarsest level is solved
// exactly: W = L^-1 of the Cholesky factor of its dense matrix is rebuilt on
// the GPU for every design (dense.cu) and each V-cycle applies W^T W.  The
// dense unknowns are ordered by node planes across the longest axis, which
// makes the matrix banded (about 3 plane sizes wide) and the factorization
// work proportional to the band.
//
// The V-cycle exists in FP64 (preconditioner of the FP64 solver) and in FP32
// (inner solver of the mixed-precision solver); the coarsest solve is FP64 in
// both.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <type_traits>
#include <vector>

#include "stencil.cuh"

namespace icarat_b200
{

void dense_spd_inverse_factor(cudaStream_t st, double *A, double *W, double *T, int n, int bw);
void dense_spd_solve(cudaStream_t st, const double *W, const double *WT, int n,
                     const double *v, double *t, const int *rowmap, double *x,
                     const int *halt = nullptr);

// Galerkin coarse operators (galerkin.cu)
__global__ void k_gal_cells_free(GridDev f, GridDev c, const double *__restrict__ E,
                                 const double *__restrict__ G,
                                 const uint8_t *__restrict__ flag, double *__restrict__ Kc);
__global__ void k_gal_cells(GridDev f, GridDev c, KeParam ke, const double *__restrict__ E,
                            const double *__restrict__ Kf, const uint8_t *__restrict__ fix_f,
                            const uint8_t *__restrict__ fix_c, const int *__restrict__ cells,
                            int ncells, double *__restrict__ Kc, double *__restrict__ lmax);
__global__ void k_gal_stencil(GridDev g, const double *__restrict__ Kc,
                              const uint8_t *__restrict__ fix, double *__restrict__ S,
                              double *__restrict__ invd);
__global__ void k_gal_coefs(int levels, const double *__restrict__ lmax, double lam1,
                            double *__restrict__ coef);
double galerkin_child_matrices(const double *ke0, double *G);
template <typename T>
void st_first_launch(cudaStream_t st, int n, const T *b, const T *invd, const double *coef,
                     T *x, T *d, const int *halt);
template <typename T>
void st_cheb_launch(cudaStream_t st, const GridDev &g, const T *S, const uint8_t *fix,
                    const T *invd, const T *b, const T *x, T *d, T *xo, const double *coef, int k,
                    const int *halt);
template <typename T>
void st_residual_launch(cudaStream_t st, const GridDev &g, const T *S, const uint8_t *fix,
                        const T *b, const T *x, T *r, const int *halt);
__global__ void k_coarse_assemble_st(GridDev g, const double *__restrict__ S,
                                     const int *__restrict__ rowmap,
                                     const int *__restrict__ colmap, int nfree,
                                     double *__restrict__ A);

// ---------------------------------------------------------------- level data
__global__ void k_coarsen_E(GridDev f, GridDev c, const double *__restrict__ Ef,
                            double *__restrict__ Ec)
{
  for(int e = blockIdx.x * blockDim.x + threadIdx.x; e < c.nelx;
      e += gridDim.x * blockDim.x)
  {
    const int I = e % c.nx, J = (e / c.nx) % c.ny, K = e / (c.nx * c.ny);
    double s = 0.0;
#pragma unroll
    for(int dz = 0; dz < 2; dz++)
#pragma unroll
      for(int dy = 0; dy < 2; dy++)
#pragma unroll
        for(int dx = 0; dx < 2; dx++)
          s += Ef[(2 * I + dx) + (long)(2 * J + dy) * f.nx +
                  (long)(2 * K + dz) * f.nx * f.ny];
    Ec[e] = 0.25 * s; // mean of 8 children x 2
  }
}

template <typename Tin, typename Tout>
__global__ void k_cast(long n, const Tin *__restrict__ in, Tout *__restrict__ out)
{
  chain_wait();
  for(long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
      i += (long)gridDim.x * blockDim.x)
    out[i] = (Tout)in[i];
}

// ---------------------------------------------------------------- transfers
// coarse b = R r  (R = P^T, 27 fine nodes per coarse node, weights 1/2^d;
// restrict_node / prolong_node in stencil.cuh)
template <typename T>
// With xc set, also the coarse level's first Chebyshev step from zero
// (k_cheb_first fused): dc = xc = inv_theta invd_c bc.
__global__ void k_restrict(GridDev f, GridDev c, const T *__restrict__ rf,
                           const uint8_t *__restrict__ fixc, T *__restrict__ bc,
                           const T *__restrict__ invd_c, T inv_theta, T *__restrict__ xc,
                           T *__restrict__ dc, const int *__restrict__ halt)
{
  chain_wait();
  if(halted(halt))
    return;
  for(int n = blockIdx.x * blockDim.x + threadIdx.x; n < c.numnp;
      n += gridDim.x * blockDim.x)
  {
    T s[3];
    restrict_node<T, false>(f, c, rf, n, s);
    const unsigned fx = fixc[n];
#pragma unroll
    for(int q = 0; q < 3; q++)
    {
      const long id = (long)q * c.numnp + n;
      const T bq = ((fx >> q) & 1u) ? T(0) : s[q];
      bc[id] = bq;
      if(xc)
      {
        const T di = inv_theta * invd_c[id] * bq;
        dc[id] = di;
        xc[id] = di;
      }
    }
  }
}

// fine x += P xc (masked)
template <typename T>
__global__ void k_prolong_add(GridDev f, GridDev c, const T *__restrict__ xc,
                              const uint8_t *__restrict__ fixf, T *__restrict__ xf,
                              const int *__restrict__ halt)
{
  chain_wait();
  if(halted(halt))
    return;
  for(int n = blockIdx.x * blockDim.x + threadIdx.x; n < f.numnp;
      n += gridDim.x * blockDim.x)
  {
    T s[3];
    prolong_node<T, false>(f, c, xc, n, s);
    const unsigned fx = fixf[n];
#pragma unroll
    for(int q = 0; q < 3; q++)
      if(!((fx >> q) & 1u))
        xf[(long)q * f.numnp + n] += s[q];
  }
}

// ---------------------------------------------------------------- smoother
// First Chebyshev step from x = 0: d = invd b / theta, x = d.
template <typename T>
__global__ void k_cheb_first(int n, const T *__restrict__ b, const T *__restrict__ invd,
                             T inv_theta, T *__restrict__ x, T *__restrict__ d,
                             const int *__restrict__ halt)
{
  chain_wait();
  if(halted(halt))
    return;
  for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
      i += gridDim.x * blockDim.x)
  {
    const T di = inv_theta * invd[i] * b[i];
    d[i] = di;
    x[i] = di;
  }
}

// One Chebyshev step: r = b - K x, d = c1 d + c2 invd r, xo = x + d.
// x and xo are distinct buffers (neighbours of x are read by other threads).
template <typename T, typename KP>
__global__ void __launch_bounds__(128)
    k_cheb_step(GridDev g, MarchPlan m, KP ke, const T *__restrict__ E,
                const uint8_t *__restrict__ fix, const T *__restrict__ invd,
                const T *__restrict__ b, const T *__restrict__ x, T *__restrict__ d,
                T *__restrict__ xo, T c1, T c2, const int *__restrict__ halt)
{
  chain_wait();
  if(halted(halt))
    return;
  for(long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < m.items;
      t += (long)gridDim.x * blockDim.x)
  {
    int i, j, k0, k1;
    if(!march_item(g, m, t, i, j, k0, k1))
      continue;
    column_Ku(g, ke, E, x, i, j, k0, k1,
              [&](int k, const T(&acc)[3], const T(&uc)[3])
              {
                const int n = i + j * g.NX + k * g.NX * g.NY;
                const unsigned f = fix[n];
#pragma unroll
                for(int q = 0; q < 3; q++)
                {
                  const long id = (long)q * g.numnp + n;
                  T dn = 0;
                  if(!((f >> q) & 1u))
                    dn = (c1 != T(0) ? c1 * d[id] : T(0)) + c2 * invd[id] * (b[id] - acc[q]);
                  d[id] = dn;
                  xo[id] = uc[q] + dn;
                }
              });
  }
}

// r = b - K x (constrained rows 0)
template <typename T, typename KP>
__global__ void __launch_bounds__(128)
    k_mg_residual(GridDev g, MarchPlan m, KP ke, const T *__restrict__ E,
                  const uint8_t *__restrict__ fix, const T *__restrict__ b,
                  const T *__restrict__ x, T *__restrict__ r, const int *__restrict__ halt)
{
  chain_wait();
  if(halted(halt))
    return;
  for(long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < m.items;
      t += (long)gridDim.x * blockDim.x)
  {
    int i, j, k0, k1;
    if(!march_item(g, m, t, i, j, k0, k1))
      continue;
    column_Ku(g, ke, E, x, i, j, k0, k1,
              [&](int k, const T(&acc)[3], const T(&)[3])
              {
                const int n = i + j * g.NX + k * g.NX * g.NY;
                const unsigned f = fix[n];
#pragma unroll
                for(int c = 0; c < 3; c++)
                  r[(long)c * g.numnp + n] =
                      ((f >> c) & 1u) ? T(0) : b[(long)c * g.numnp + n] - acc[c];
              });
  }
}

// ---------------------------------------------------------------- coarse
// Dense coarse matrix, one thread per free row (fixed summation order).
__global__ void k_coarse_assemble(GridDev g, KeParam ke, const double *__restrict__ E,
                                  const int *__restrict__ rowmap,
                                  const int *__restrict__ colmap, int nfree,
                                  double *__restrict__ A)
{
  for(int r = blockIdx.x * blockDim.x + threadIdx.x; r < nfree;
      r += gridDim.x * blockDim.x)
  {
    double *row = A + (long)r * nfree; // zeroed by the caller
    const int full = rowmap[r];        // component-major index c * numnp + n
    const int n = full % g.numnp, c = full / g.numnp;
    const int i = n % g.NX, j = (n / g.NX) % g.NY, k = n / (g.NX * g.NY);
    for(int sz = 0; sz < 2; sz++)
      for(int sy = 0; sy < 2; sy++)
        for(int sx = 0; sx < 2; sx++)
        {
          const int ei = i - 1 + sx, ej = j - 1 + sy, ek = k - 1 + sz;
          if(ei < 0 || ei >= g.nx || ej < 0 || ej >= g.ny || ek < 0 || ek >= g.nz)
            continue;
          const double e = E[ei + (long)ej * g.nx + (long)ek * g.nx * g.ny];
          const int a = local_node(1 - sx, 1 - sy, 1 - sz);
          for(int bz = 0; bz < 2; bz++)
            for(int by = 0; by < 2; by++)
              for(int bx = 0; bx < 2; bx++)
              {
                const int b = local_node(bx, by, bz);
                const long m = (ei + bx) + (long)(ej + by) * g.NX +
                               (long)(ek + bz) * g.NX * g.NY;
                for(int d = 0; d < 3; d++)
                {
                  const int col = colmap[3 * m + d];
                  if(col >= 0)
                    row[col] += e * ke.k[(3 * a + c) * 24 + 3 * b + d];
                }
              }
        }
  }
}

// free coarse components of b (any precision) into the dense solve's vector
template <typename T>
__global__ void k_coarse_gather(int nfree, const int *__restrict__ rowmap,
                                const T *__restrict__ b, double *__restrict__ v,
                                const int *__restrict__ halt)
{
  chain_wait();
  if(halted(halt))
    return;
  for(int r = blockIdx.x * blockDim.x + threadIdx.x; r < nfree;
      r += gridDim.x * blockDim.x)
    v[r] = (double)b[rowmap[r]];
}

// ---------------------------------------------------------------- driver
static GridDev make_grid(int nx, int ny, int nz)
{
  return GridDev{nx, ny, nz, nx + 1, ny + 1, nz + 1, (nx + 1) * (ny + 1) * (nz + 1),
                 nx * ny * nz};
}

static int blocks_for(long n, int t)
{
  long b = (n + t - 1) / t;
  return b < 1 ? 1 : (b > 65535L * 16 ? 65535 * 16 : (int)b);
}

// level buffers of one precision
template <typename T> struct LevelBuf;
template <> struct LevelBuf<double>
{
  static double *E(MgLevel &L) { return L.E; }
  static double *invd(MgLevel &L) { return L.invd; }
  static double *x(MgLevel &L) { return L.x; }
  static double *b(MgLevel &L) { return L.b; }
  static double *r(MgLevel &L) { return L.r; }
  static double *t(MgLevel &L) { return L.t; }
  static double *S(MgLevel &L) { return L.S; }
  static const KeParam &ke(icarat_ctx *c) { return c->ke0; }
};
template <> struct LevelBuf<float>
{
  static float *E(MgLevel &L) { return L.E32; }
  static float *invd(MgLevel &L) { return L.invd32; }
  static float *x(MgLevel &L) { return L.x32; }
  static float *b(MgLevel &L) { return L.b32; }
  static float *r(MgLevel &L) { return L.r32; }
  static float *t(MgLevel &L) { return L.t32; }
  static float *S(MgLevel &L) { return L.S32; }
  static const KeParamF &ke(icarat_ctx *c) { return c->ke0f; }
};

void mg_free(icarat_ctx *c)
{
  for(size_t l = 0; l < c->mg.size(); l++)
  {
    MgLevel &L = c->mg[l];
    if(l > 0)
    {
      dfree(L.E);
      dfree(L.fix);
      dfree(L.invd);
      dfree(L.E32);
    }
    for(void *p : {(void *)L.x, (void *)L.b, (void *)L.r, (void *)L.t, (void *)L.invd32,
                   (void *)L.x32, (void *)L.b32, (void *)L.r32, (void *)L.t32, (void *)L.Kc,
                   (void *)L.S, (void *)L.S32})
      dfree(p);
  }
  c->mg.clear();
  dfree(c->gal_lmax);
  c->gal_lmax = nullptr;
  dfree(c->gal_G);
  c->gal_G = nullptr;
  dfree(c->gal_flag1);
  c->gal_flag1 = nullptr;
  dfree(c->gal_cells1);
  c->gal_cells1 = nullptr;
  c->gal_ncells1 = 0;
  c->gal_coef = nullptr; // part of the gal_lmax allocation
  c->mg_galerkin = 0;
  CoarseSolver &C = c->coarse;
  if(C.side)
    cudaStreamSynchronize(C.side); // a lagged factorization may still run
  for(int b = 0; b < 2; b++)
  {
    if(C.setup[b])
      cudaGraphExecDestroy(C.setup[b]);
    if(C.factor[b])
      cudaGraphExecDestroy(C.factor[b]);
    if(C.ev_factor[b])
      cudaEventDestroy(C.ev_factor[b]);
    dfree(C.A[b]);
    dfree(C.W[b]);
    dfree(C.work[b]);
  }
  if(C.levels)
    cudaGraphExecDestroy(C.levels);
  if(C.ev_levels)
    cudaEventDestroy(C.ev_levels);
  if(C.side)
    cudaStreamDestroy(C.side);
  dfree(C.map);
  dfree(C.vin);
  dfree(C.vout);
  c->coarse = CoarseSolver{};
  c->mg_built_levels = 0;
}

static float *falloc(size_t n)
{
  void *p = nullptr;
  cudaError_t e = cudaMalloc(&p, (n ? n : 1) * sizeof(float));
  if(e != cudaSuccess)
    throw Error{ICARAT_ERR_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e)};
  return static_cast<float *>(p);
}

static void allocate_levels(icarat_ctx *c, int levels)
{
  release_graphs(c); // captured solver graphs hold pointers to level arrays
  mg_free(c);
  int nx = c->nx, ny = c->ny, nz = c->nz;
  for(int l = 0; l < levels; l++)
  {
    if(l > 0)
    {
      IREQUIRE(nx % 2 == 0 && ny % 2 == 0 && nz % 2 == 0, ICARAT_ERR_UNSUPPORTED,
               "multigrid needs divisions divisible by 2^(levels-1)");
      nx /= 2;
      ny /= 2;
      nz /= 2;
    }
    MgLevel L;
    L.g = make_grid(nx, ny, nz);
    const size_t nv = 3 * (size_t)L.g.numnp;
    if(l == 0)
    {
      L.E = c->d_E;
      L.E32 = c->d_E32;
      L.fix = c->d_fix;
      L.invd = c->d_invd;
    }
    else
    {
      L.E = dalloc(L.g.nelx);
      L.E32 = falloc(L.g.nelx);
      ICK(cudaMalloc(&L.fix, L.g.numnp));
      L.invd = dalloc(nv);
    }
    if(l > 0 && c->mg_galerkin_req)
    {
      L.Kc = dalloc(576 * (size_t)L.g.nelx);
      L.S = dalloc(126 * (size_t)L.g.numnp);
      L.S32 = falloc(126 * (size_t)L.g.numnp);
    }
    L.x = dalloc(nv);
    L.b = dalloc(nv);
    L.r = dalloc(nv);
    L.t = dalloc(nv);
    L.invd32 = falloc(nv);
    L.x32 = falloc(nv);
    L.b32 = falloc(nv);
    L.r32 = falloc(nv);
    L.t32 = falloc(nv);
    c->mg.push_back(L);
  }
  if(c->mg_galerkin_req)
  {
    // per level: the Chebyshev bound, then kGalCoef coefficients
    c->gal_lmax = dalloc((size_t)levels * (1 + kGalCoef));
    c->gal_coef = c->gal_lmax + levels;
    std::vector<double> G(8 * 576);
    c->gal_lam1 = 1.001 * galerkin_child_matrices(c->ke0.k, G.data());
    c->gal_G = dalloc(G.size());
    ICK(cudaMemcpy(c->gal_G, G.data(), sizeof(double) * G.size(), cudaMemcpyHostToDevice));
    // level-1 cells with a constrained child node (fixed for the context):
    // they take the general cell kernel, the others the free form
    const GridDev f0 = c->mg[0].g, g1 = c->mg[1].g;
    std::vector<uint8_t> flag(g1.nelx, 0);
    std::vector<int> cells;
    for(int cell = 0; cell < g1.nelx; cell++)
    {
      const int CI = cell % g1.nx, CJ = (cell / g1.nx) % g1.ny, CK = cell / (g1.nx * g1.ny);
      for(int t = 0; t < 27 && !flag[cell]; t++)
      {
        const int fx = t % 3, fy = (t / 3) % 3, fz = t / 9;
        if(c->fix_h[(2 * CI + fx) + (2L * CJ + fy) * f0.NX + (2L * CK + fz) * f0.NX * f0.NY])
          flag[cell] = 1;
      }
      if(flag[cell])
        cells.push_back(cell);
    }
    ICK(cudaMalloc(&c->gal_flag1, g1.nelx));
    ICK(cudaMemcpy(c->gal_flag1, flag.data(), g1.nelx, cudaMemcpyHostToDevice));
    c->gal_ncells1 = (int)cells.size();
    ICK(cudaMalloc(&c->gal_cells1, sizeof(int) * std::max<size_t>(1, cells.size())));
    if(!cells.empty())
      ICK(cudaMemcpy(c->gal_cells1, cells.data(), sizeof(int) * cells.size(),
                     cudaMemcpyHostToDevice));
  }
  c->mg_galerkin = c->mg_galerkin_req;
  // coarse constraint pattern on the host (fixed for the context)
  std::vector<uint8_t> fix = c->fix_h;
  GridDev gf = c->mg[0].g;
  for(int l = 1; l < levels; l++)
  {
    GridDev gc = c->mg[l].g;
    std::vector<uint8_t> fc(gc.numnp);
    for(int n = 0; n < gc.numnp; n++)
    {
      int I = n % gc.NX, J = (n / gc.NX) % gc.NY, K = n / (gc.NX * gc.NY);
      fc[n] = fix[2 * I + (long)2 * J * gf.NX + (long)2 * K * gf.NX * gf.NY];
    }
    ICK(cudaMemcpy(c->mg[l].fix, fc.data(), gc.numnp, cudaMemcpyHostToDevice));
    fix.swap(fc);
    gf = gc;
  }
  // dense coarse system: unknowns ordered by node planes across the longest
  // axis (nodes within a plane, then the 3 components), so that the matrix
  // is banded (a node couples to the planes either side only) with the
  // narrowest band
  GridDev gc = c->mg[levels - 1].g;
  std::vector<int> rowmap, colmap(3 * (size_t)gc.numnp, -1);
  const int ext[3] = {gc.NX, gc.NY, gc.NZ};
  int ax[3] = {0, 1, 2}; // slowest .. fastest
  std::stable_sort(ax, ax + 3, [&](int p, int q) { return ext[p] > ext[q]; });
  int id[3];
  for(id[ax[0]] = 0; id[ax[0]] < ext[ax[0]]; id[ax[0]]++)
    for(id[ax[1]] = 0; id[ax[1]] < ext[ax[1]]; id[ax[1]]++)
      for(id[ax[2]] = 0; id[ax[2]] < ext[ax[2]]; id[ax[2]]++)
      {
        const int n = id[0] + gc.NX * (id[1] + gc.NY * id[2]);
        for(int q = 0; q < 3; q++)
          if(!((fix[n] >> q) & 1u))
          {
            colmap[3 * (size_t)n + q] = (int)rowmap.size(); // node-major lookup table
            rowmap.push_back(q * gc.numnp + n);             // component-major vector index
          }
      }
  const int nf = (int)rowmap.size();
  int bw = 0; // largest index distance of two coupled unknowns
  for(int n = 0; n < gc.numnp; n++)
  {
    const int I = n % gc.NX, J = (n / gc.NX) % gc.NY, K = n / (gc.NX * gc.NY);
    for(int dk = -1; dk <= 1; dk++)
      for(int dj = -1; dj <= 1; dj++)
        for(int di = -1; di <= 1; di++)
        {
          const int i2 = I + di, j2 = J + dj, k2 = K + dk;
          if(i2 < 0 || j2 < 0 || k2 < 0 || i2 >= gc.NX || j2 >= gc.NY || k2 >= gc.NZ)
            continue;
          const int n2 = i2 + gc.NX * (j2 + gc.NY * k2);
          for(int q = 0; q < 3; q++)
            for(int q2 = 0; q2 < 3; q2++)
            {
              const int u = colmap[3 * (size_t)n + q], v = colmap[3 * (size_t)n2 + q2];
              if(u >= 0 && v >= 0)
                bw = std::max(bw, std::abs(u - v));
            }
        }
  }
  c->coarse.bw = bw;
  IREQUIRE((double)nf * nf * 8.0 * 3 < 6.0e9, ICARAT_ERR_UNSUPPORTED,
           "coarsest multigrid level too large for the dense solve; add levels");
  c->coarse.n = nf;
  ICK(cudaMalloc(&c->coarse.map, sizeof(int) * (rowmap.size() + colmap.size() + 1)));
  if(nf > 0)
    ICK(cudaMemcpy(c->coarse.map, rowmap.data(), sizeof(int) * nf,
                   cudaMemcpyHostToDevice));
  ICK(cudaMemcpy(c->coarse.map + nf, colmap.data(), sizeof(int) * colmap.size(),
                 cudaMemcpyHostToDevice));
  c->coarse.A[0] = dalloc((size_t)nf * nf);
  c->coarse.W[0] = dalloc((size_t)nf * nf);
  c->coarse.work[0] = dalloc((size_t)nf * nf);
  c->coarse.vin = dalloc(nf);
  c->coarse.vout = dalloc(nf);
  c->mg_built_levels = levels;
}

// Everything on the levels that depends on the design: coarse moduli and
// Jacobi diagonals (and their FP32 copies).
static void enqueue_levels(icarat_ctx *c, int levels, cudaStream_t st)
{
  if(c->mg_galerkin)
    ICK(cudaMemsetAsync(c->gal_lmax, 0, sizeof(double) * levels, st));
  for(int l = 0; l < levels; l++)
  {
    MgLevel &L = c->mg[l];
    if(l > 0)
    {
      const MgLevel &F = c->mg[l - 1];
      note_launch();
      k_coarsen_E<<<blocks_for(L.g.nelx, 256), 256, 0, st>>>(F.g, L.g, F.E, L.E);
    }
    if(l > 0 && c->mg_galerkin)
    {
      // Galerkin: cell matrices from the level above, the node stencil, the
      // Jacobi diagonal from it, the FP32 copies
      const MgLevel &F = c->mg[l - 1];
      if(l == 1)
      {
        note_launch();
        k_gal_cells_free<<<blocks_for(576L * L.g.nelx, 256), 256, 0, st>>>(
            F.g, L.g, F.E, c->gal_G, c->gal_flag1, L.Kc);
        if(c->gal_ncells1 > 0)
        {
          note_launch();
          k_gal_cells<<<c->gal_ncells1, 128, 0, st>>>(F.g, L.g, c->ke0, F.E, nullptr, F.fix,
                                                      L.fix, c->gal_cells1, c->gal_ncells1, L.Kc,
                                                      c->gal_lmax + l);
        }
      }
      else
      {
        note_launch();
        k_gal_cells<<<L.g.nelx, 128, 0, st>>>(F.g, L.g, c->ke0, F.E, F.Kc, F.fix, L.fix, nullptr,
                                              L.g.nelx, L.Kc, c->gal_lmax + l);
      }
      note_launch(2);
      k_gal_stencil<<<blocks_for(14L * L.g.numnp, 256), 256, 0, st>>>(L.g, L.Kc, L.fix, L.S,
                                                                      L.invd);
      k_cast<<<blocks_for(126L * L.g.numnp, 256), 256, 0, st>>>(126L * L.g.numnp, L.S, L.S32);
    }
    else
      launch_diag(c, L.g, L.E, L.fix, L.invd, st);
    if(l > 0) // the finest FP32 moduli come with the design
    {
      note_launch();
      k_cast<<<blocks_for(L.g.nelx, 256), 256, 0, st>>>((long)L.g.nelx, L.E, L.E32);
    }
    note_launch();
    k_cast<<<blocks_for(3L * L.g.numnp, 256), 256, 0, st>>>(3L * L.g.numnp, L.invd,
                                                           L.invd32);
  }
  if(c->mg_galerkin)
  {
    note_launch();
    k_gal_coefs<<<1, 32, 0, st>>>(levels, c->gal_lmax, c->gal_lam1, c->gal_coef);
  }
}

// The dense coarsest matrix of the current coarsest moduli and W = L^-1 of
// its Cholesky factor, into factor buffer b.
static void enqueue_factor(icarat_ctx *c, int b, cudaStream_t st)
{
  const MgLevel &C = c->mg.back();
  const int n = c->coarse.n;
  if(n == 0)
    return;
  ICK(cudaMemsetAsync(c->coarse.A[b], 0, sizeof(double) * (size_t)n * n, st));
  note_launch();
  if(c->mg_galerkin)
    k_coarse_assemble_st<<<blocks_for(n, 64), 64, 0, st>>>(C.g, C.S, c->coarse.map,
                                                           c->coarse.map + n, n,
                                                           c->coarse.A[b]);
  else
    k_coarse_assemble<<<blocks_for(n, 64), 64, 0, st>>>(C.g, c->ke0, C.E, c->coarse.map,
                                                       c->coarse.map + n, n, c->coarse.A[b]);
  ICK(cudaGetLastError());
  dense_spd_inverse_factor(st, c->coarse.A[b], c->coarse.W[b], c->coarse.work[b], n,
                           c->coarse.bw);
}

// ||b - K_c x|| / ||b|| of the coarsest dense solve for a fixed right-hand
// side (a check of the factorization), K_c applied by the coarsest level's
// stencil.
double mg_coarse_check(icarat_ctx *c, int levels, int *n_coarse)
{
  mg_setup(c, levels);
  const MgLevel &C = c->mg.back();
  const int n = c->coarse.n;
  if(n_coarse)
    *n_coarse = n;
  if(n == 0)
    return 0.0;
  const size_t nv = 3 * (size_t)C.g.numnp;
  std::vector<int> rowmap(n);
  std::vector<double> b(n), y(nv);
  for(int i = 0; i < n; i++)
    b[i] = 1.0 + (i % 7) / 7.0;
  ICK(cudaStreamSynchronize(c->stream));
  ICK(cudaMemcpy(rowmap.data(), c->coarse.map, sizeof(int) * n, cudaMemcpyDeviceToHost));
  ICK(cudaMemcpy(c->coarse.vin, b.data(), sizeof(double) * n, cudaMemcpyHostToDevice));
  ICK(cudaMemsetAsync(C.x, 0, sizeof(double) * nv, c->stream));
  dense_spd_solve(c->stream, c->coarse.W[c->coarse.cur], c->coarse.work[c->coarse.cur], n,
                  c->coarse.vin, c->coarse.vout, c->coarse.map, C.x);
  if(c->mg_galerkin)
  {
    // A x with the stencil: the residual of b = 0 is -A x
    ICK(cudaMemsetAsync(C.b, 0, sizeof(double) * nv, c->stream));
    st_residual_launch<double>(c->stream, C.g, C.S, C.fix, C.b, C.x, C.t, nullptr);
    ICK(cudaStreamSynchronize(c->stream));
    std::vector<double> tmp(nv);
    ICK(cudaMemcpy(tmp.data(), C.t, sizeof(double) * nv, cudaMemcpyDeviceToHost));
    for(double &v : tmp)
      v = -v;
    ICK(cudaMemcpy(C.t, tmp.data(), sizeof(double) * nv, cudaMemcpyHostToDevice));
  }
  else
    launch_apply_K(c, C.g, C.E, C.fix, C.x, C.t, nullptr);
  ICK(cudaMemcpyAsync(y.data(), C.t, sizeof(double) * nv, cudaMemcpyDeviceToHost, c->stream));
  ICK(cudaStreamSynchronize(c->stream));
  double rr = 0.0, bb = 0.0;
  for(int i = 0; i < n; i++)
  {
    const double r = b[i] - y[rowmap[i]];
    rr += r * r;
    bb += b[i] * b[i];
  }
  return std::sqrt(rr / bb);
}

// y = A_level x on the host (component-major vectors of the level's 3 numnp
// entries): the operator the V-cycle applies on that level for the options'
// levels and coarse operators (constrained rows 0).
void mg_level_apply(icarat_ctx *c, const icarat_solve_opts *o, int level, const double *x,
                    double *y)
{
  const int levels = o->mg_levels > 0 ? o->mg_levels : 4;
  IREQUIRE(o->coarse_op == ICARAT_COARSE_REDISCRETISED || o->coarse_op == ICARAT_COARSE_GALERKIN,
           ICARAT_ERR_ARG, "coarse_op must be ICARAT_COARSE_REDISCRETISED or _GALERKIN");
  IREQUIRE(level >= 0 && level < levels, ICARAT_ERR_ARG, "level out of range");
  c->mg_galerkin_req = o->coarse_op == ICARAT_COARSE_GALERKIN ? 1 : 0;
  mg_setup(c, levels);
  MgLevel &L = c->mg[level];
  const size_t nv = 3 * (size_t)L.g.numnp;
  ICK(cudaMemcpyAsync(L.x, x, sizeof(double) * nv, cudaMemcpyHostToDevice, c->stream));
  if(level > 0 && c->mg_galerkin)
  {
    ICK(cudaMemsetAsync(L.b, 0, sizeof(double) * nv, c->stream));
    st_residual_launch<double>(c->stream, L.g, L.S, L.fix, L.b, L.x, L.t, nullptr);
    ICK(cudaMemcpyAsync(y, L.t, sizeof(double) * nv, cudaMemcpyDeviceToHost, c->stream));
    ICK(cudaStreamSynchronize(c->stream));
    for(size_t i = 0; i < nv; i++)
      y[i] = -y[i];
    return;
  }
  launch_apply_K(c, L.g, L.E, L.fix, L.x, L.t, nullptr);
  ICK(cudaMemcpyAsync(y, L.t, sizeof(double) * nv, cudaMemcpyDeviceToHost, c->stream));
  ICK(cudaStreamSynchronize(c->stream));
}

// Captures what f enqueues on stream st into an instantiated graph.
template <typename F>
static cudaGraphExec_t capture(cudaStream_t st, int &kernels, F f)
{
  cudaGraph_t graph;
  ICK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
  set_capturing(true);
  try
  {
    f();
  }
  catch(...)
  {
    set_capturing(false);
    cudaStreamEndCapture(st, &graph);
    throw;
  }
  set_capturing(false);
  ICK(cudaStreamEndCapture(st, &graph));
  size_t nn = 0;
  ICK(cudaGraphGetNodes(graph, nullptr, &nn));
  std::vector<cudaGraphNode_t> nodes(nn);
  ICK(cudaGraphGetNodes(graph, nodes.data(), &nn));
  kernels = 0;
  for(auto nd : nodes)
  {
    cudaGraphNodeType t;
    ICK(cudaGraphNodeGetType(nd, &t));
    kernels += (t == cudaGraphNodeTypeKernel) ? 1 : 0;
  }
  cudaGraphExec_t exec;
  ICK(cudaGraphInstantiate(&exec, graph, 0));
  cudaGraphDestroy(graph);
  return exec;
}

// Coarse operators and the dense inverse for the current design.  The fixed
// launch sequences are captured once per hierarchy into CUDA graphs and
// replayed for every new design.
//
// Lagged set-up (factor reuse across design iterations): the levels of the
// new design are built on the context's stream as usual, but its coarsest
// factor goes into the other buffer on a side stream, overlapped with the
// solve, which keeps the factor of the previous design; the next set-up
// waits for it and switches buffers.  The coarse correction then belongs to
// a slightly different operator, which costs at most a few iterations while
// the design changes slowly; the solve's stopping test is unchanged.
void mg_setup(icarat_ctx *c, int levels, bool lag)
{
  IREQUIRE(levels >= 2 && levels <= 12, ICARAT_ERR_ARG, "mg_levels must be in [2, 12]");
  if((int)c->mg.size() != levels || c->mg_galerkin != c->mg_galerkin_req)
    allocate_levels(c, levels);
  else if(c->mg_version == c->design_version)
  {
    // operators of this design are built; its lagged factor replaces the
    // previous design's once it has finished (a synchronous request waits
    // for it)
    CoarseSolver &C = c->coarse;
    if(C.pending >= 0 && (!lag || cudaEventQuery(C.ev_factor[C.pending]) == cudaSuccess))
    {
      ICK(cudaStreamWaitEvent(c->stream, C.ev_factor[C.pending], 0));
      C.cur = C.pending;
      C.pending = -1;
    }
    return;
  }
  c->mg_version = c->design_version;
  CoarseSolver &C = c->coarse;
  if(C.pending >= 0)
  {
    // the previous design's factor (lagged) is needed now, and its inputs
    // (the coarsest moduli) are about to be overwritten
    ICK(cudaStreamWaitEvent(c->stream, C.ev_factor[C.pending], 0));
    C.cur = C.pending;
    C.pending = -1;
  }
  if(!lag || !C.have || C.n == 0)
  {
    const int b = C.cur;
    if(!C.setup[b])
      C.setup[b] = capture(c->stream, C.setup_kernels, [&] {
        enqueue_levels(c, levels, c->stream);
        enqueue_factor(c, b, c->stream);
      });
    ICK(cudaGraphLaunch(C.setup[b], c->stream));
    note_launch(C.setup_kernels);
    C.have = true;
    return;
  }
  const int nb = 1 - C.cur;
  if(!C.A[nb])
  {
    const size_t nn = (size_t)C.n * C.n;
    C.A[nb] = dalloc(nn);
    C.W[nb] = dalloc(nn);
    C.work[nb] = dalloc(nn);
  }
  if(!C.side)
  {
    ICK(cudaStreamCreateWithFlags(&C.side, cudaStreamNonBlocking));
    ICK(cudaEventCreateWithFlags(&C.ev_levels, cudaEventDisableTiming));
    for(int b = 0; b < 2; b++)
      ICK(cudaEventCreateWithFlags(&C.ev_factor[b], cudaEventDisableTiming));
  }
  if(!C.levels)
    C.levels = capture(c->stream, C.levels_kernels, [&] { enqueue_levels(c, levels, c->stream); });
  if(!C.factor[nb])
    C.factor[nb] = capture(C.side, C.factor_kernels, [&] { enqueue_factor(c, nb, C.side); });
  ICK(cudaGraphLaunch(C.levels, c->stream));
  note_launch(C.levels_kernels);
  ICK(cudaEventRecord(C.ev_levels, c->stream));
  ICK(cudaStreamWaitEvent(C.side, C.ev_levels, 0));
  ICK(cudaGraphLaunch(C.factor[nb], C.side));
  note_launch(C.factor_kernels);
  ICK(cudaEventRecord(C.ev_factor[nb], C.side));
  C.pending = nb;
}

void mg_join(icarat_ctx *c)
{
  if(c->coarse.pending >= 0)
    ICK(cudaStreamWaitEvent(c->stream, c->coarse.ev_factor[c->coarse.pending], 0));
}

// the finest level of the FP32 V-cycle may run on the tensor-core operator
template <typename T> static bool tc_level(icarat_ctx *c, int lvl)
{
  return std::is_same<T, float>::value && lvl == 0 &&
         (c->mx_fine_op == ICARAT_OP_TC_BF16X3 || c->mx_fine_op == ICARAT_OP_TC_BF16);
}

// one Chebyshev step d = c1 d + c2 invd (b - K x), xo = x + d on level lvl
template <typename T>
static void cheb_step(icarat_ctx *c, MgLevel &L, int lvl, const T *b, const T *x, T *d, T *xo,
                      double c1, double c2)
{
  using B = LevelBuf<T>;
  if(tc_level<T>(c, lvl))
  {
    TcArgs a;
    a.g = L.g;
    a.E = reinterpret_cast<const float *>(B::E(L));
    a.fix = L.fix;
    a.u = reinterpret_cast<const float *>(x);
    a.y = reinterpret_cast<float *>(xo);
    a.b = reinterpret_cast<const float *>(b);
    a.invd = reinterpret_cast<const float *>(B::invd(L));
    a.d = reinterpret_cast<float *>(d);
    a.c1 = (float)c1;
    a.c2 = (float)c2;
    a.halt = c->mg_halt;
    launch_ku_tc(c, TC_CHEB, c->mx_fine_op == ICARAT_OP_TC_BF16X3 ? 3 : 1, a, c->stream);
    return;
  }
  if constexpr(std::is_same<T, double>::value)
    if(use_dmma(c, L.g))
    {
      DmArgs a;
      a.g = L.g;
      a.E = B::E(L);
      a.fix = L.fix;
      a.u = x;
      a.y = xo;
      a.b = b;
      a.invd = B::invd(L);
      a.d = d;
      a.c1 = c1;
      a.c2 = c2;
      a.halt = c->mg_halt;
      launch_ku_dmma(c, TC_CHEB, a, c->stream);
      return;
    }
  int blocks;
  const MarchPlan m =
      march_launch(L.g, (const void *)k_cheb_step<T, typename KeOf<T>::type>, 128,
                   c->sm_count, blocks);
  note_launch();
  launch_chained(k_cheb_step<T, typename KeOf<T>::type>, blocks, 128, 0, c->stream, L.g, m,
                 B::ke(c), B::E(L), L.fix, B::invd(L), b, x, d, xo, T(c1), T(c2), c->mg_halt);
}

// r = b - K x on level lvl
template <typename T>
static void mg_residual(icarat_ctx *c, MgLevel &L, int lvl, const T *b, const T *x, T *r)
{
  using B = LevelBuf<T>;
  if(lvl > 0 && c->mg_galerkin)
  {
    st_residual_launch<T>(c->stream, L.g, B::S(L), L.fix, b, x, r, c->mg_halt);
    return;
  }
  if(tc_level<T>(c, lvl))
  {
    TcArgs a;
    a.g = L.g;
    a.E = reinterpret_cast<const float *>(B::E(L));
    a.fix = L.fix;
    a.u = reinterpret_cast<const float *>(x);
    a.y = reinterpret_cast<float *>(r);
    a.b = reinterpret_cast<const float *>(b);
    a.halt = c->mg_halt;
    launch_ku_tc(c, TC_RESID, c->mx_fine_op == ICARAT_OP_TC_BF16X3 ? 3 : 1, a, c->stream);
    return;
  }
  if constexpr(std::is_same<T, double>::value)
    if(use_dmma(c, L.g))
    {
      DmArgs a;
      a.g = L.g;
      a.E = B::E(L);
      a.fix = L.fix;
      a.u = x;
      a.y = r;
      a.b = b;
      a.halt = c->mg_halt;
      launch_ku_dmma(c, TC_RESID, a, c->stream);
      return;
    }
  int blocks;
  const MarchPlan m =
      march_launch(L.g, (const void *)k_mg_residual<T, typename KeOf<T>::type>, 128,
                   c->sm_count, blocks);
  note_launch();
  launch_chained(k_mg_residual<T, typename KeOf<T>::type>, blocks, 128, 0, c->stream, L.g, m,
                 B::ke(c), B::E(L), L.fix, b, x, r, c->mg_halt);
}

// Chebyshev smoothing of K x = b on level lvl, deg steps.  from_zero: x = 0
// on entry (the first step needs no product).
template <typename T>
static void smooth(icarat_ctx *c, MgLevel &L, int lvl, const T *b, int deg, bool from_zero,
                   bool first_done = false)
{
  using B = LevelBuf<T>;
  if(lvl > 0 && c->mg_galerkin)
  {
    // the same Chebyshev sequence with the level's own bound: coefficients
    // from the device (computed at set-up from the design's cell matrices)
    IREQUIRE(deg <= (kGalCoef + 1) / 2, ICARAT_ERR_ARG,
             "mg_smooth too large for the Galerkin coarse levels");
    const double *coef = c->gal_coef + (size_t)lvl * kGalCoef;
    const int nv = 3 * L.g.numnp;
    T *x = B::x(L), *xo = B::t(L), *d = B::r(L);
    if(from_zero)
      st_first_launch<T>(c->stream, nv, b, B::invd(L), coef, x, d, c->mg_halt);
    else
    {
      st_cheb_launch<T>(c->stream, L.g, B::S(L), L.fix, B::invd(L), b, x, d, xo, coef, 0,
                        c->mg_halt);
      std::swap(x, xo);
    }
    for(int k = 1; k < deg; k++)
    {
      st_cheb_launch<T>(c->stream, L.g, B::S(L), L.fix, B::invd(L), b, x, d, xo, coef, k,
                        c->mg_halt);
      std::swap(x, xo);
    }
    if(x != B::x(L))
      ICK(cudaMemcpyAsync(B::x(L), x, sizeof(T) * nv, cudaMemcpyDeviceToDevice, c->stream));
    return;
  }
  const double lmax = c->lam_max_dk;
  const double lmin = 0.1 * lmax;
  const double theta = 0.5 * (lmax + lmin), delta = 0.5 * (lmax - lmin);
  const double sigma = theta / delta;
  double rho_old = 1.0 / sigma;
  const int nv = 3 * L.g.numnp;
  T *x = B::x(L), *xo = B::t(L), *d = B::r(L);
  int k0 = 0;
  if(from_zero)
  {
    if(!first_done) // else the restriction that produced b took this step
    {
      note_launch();
      launch_chained(k_cheb_first<T>, blocks_for(nv, 256), 256, 0, c->stream, nv, b,
                     B::invd(L), T(1.0 / theta), x, d, c->mg_halt);
    }
    k0 = 1;
  }
  else
  {
    // first step from the current x: d = invd (b - K x) / theta
    cheb_step<T>(c, L, lvl, b, x, d, xo, 0.0, 1.0 / theta);
    std::swap(x, xo);
    k0 = 1;
  }
  for(int k = k0; k < deg; k++)
  {
    const double rho = 1.0 / (2.0 * sigma - rho_old);
    cheb_step<T>(c, L, lvl, b, x, d, xo, rho * rho_old, 2.0 * rho / delta);
    std::swap(x, xo);
    rho_old = rho;
  }
  if(x != B::x(L))
    ICK(cudaMemcpyAsync(B::x(L), x, sizeof(T) * nv, cudaMemcpyDeviceToDevice, c->stream));
}

template <typename T>
static void vcycle(icarat_ctx *c, int l, const T *b, int deg, bool first_done = false)
{
  using B = LevelBuf<T>;
  MgLevel &L = c->mg[l];
  const int levels = (int)c->mg.size();
  if(l == levels - 1)
  {
    const int n = c->coarse.n;
    ICK(cudaMemsetAsync(L.x, 0, sizeof(double) * 3 * L.g.numnp, c->stream));
    if(n > 0)
    {
      note_launch();
      launch_chained(k_coarse_gather<T>, blocks_for(n, 256), 256, 0, c->stream, n,
                     c->coarse.map, b, c->coarse.vin, c->mg_halt);
      dense_spd_solve(c->stream, c->coarse.W[c->coarse.cur], c->coarse.work[c->coarse.cur],
                      n, c->coarse.vin, c->coarse.vout, c->coarse.map, L.x, c->mg_halt);
    }
    if(!std::is_same<T, double>::value)
    {
      note_launch();
      launch_chained(k_cast<double, T>, blocks_for(3L * L.g.numnp, 256), 256, 0, c->stream,
                     3L * L.g.numnp, L.x, B::x(L));
    }
    return;
  }
  MgLevel &C = c->mg[l + 1];
  smooth<T>(c, L, l, b, deg, true, first_done);
  // residual into r (smooth() used r as scratch; done with it now)
  mg_residual<T>(c, L, l, b, B::x(L), B::r(L));
  // the coarse level's first smoothing step rides on the restriction when
  // that level is smoothed with the shared rediscretised bound
  const bool fuse = l + 1 < levels - 1 && !c->mg_galerkin;
  const double lm = c->lam_max_dk, theta = 0.5 * (lm + 0.1 * lm);
  note_launch();
  launch_chained(k_restrict<T>, blocks_for(C.g.numnp, 128), 128, 0, c->stream, L.g, C.g,
                 B::r(L), C.fix, B::b(C), B::invd(C), T(1.0 / theta),
                 fuse ? B::x(C) : (T *)nullptr, B::r(C), c->mg_halt);
  vcycle<T>(c, l + 1, B::b(C), deg, fuse);
  note_launch();
  launch_chained(k_prolong_add<T>, blocks_for(L.g.numnp, 128), 128, 0, c->stream, L.g, C.g,
                 B::x(C), L.fix, B::x(L), c->mg_halt);
  smooth<T>(c, L, l, b, deg, false);
}

void mg_vcycle(icarat_ctx *c, const double *r, double *z, int deg, bool first_done)
{
  vcycle<double>(c, 0, r, deg, first_done);
  if(z)
    ICK(cudaMemcpyAsync(z, c->mg[0].x, sizeof(double) * c->neq, cudaMemcpyDeviceToDevice,
                        c->stream));
  ICK(cudaGetLastError());
}

void mg_vcycle_f32(icarat_ctx *c, const float *r, float *z, int deg)
{
  vcycle<float>(c, 0, r, deg);
  if(z)
    ICK(cudaMemcpyAsync(z, c->mg[0].x32, sizeof(float) * c->neq, cudaMemcpyDeviceToDevice,
                        c->stream));
  ICK(cudaGetLastError());
}

} // namespace icarat_b200
