// Helmholtz PDE density filter (FilterHelmholtz<E,N>,
// src/optimization/filter_helm.hpp) on the voxel grid.
//
// The reference assembles, per element and Gauss point (makeKeFint,
// :179-223), Ke += (N N^T + B^T (R / (2 sqrt 3))^2 I B) jac and
// fe += s N jac (fe /= ipmax for the sensitivity call), solves the nodal
// scalar system K val = F with "Eigen_CG" (a Jacobi-preconditioned CG,
// solvers.cpp:63-91, tolerance 1e-10 and 10000 iterations by default,
// solvers.hpp:89-90) and maps back per element (divideToElement, :225-257):
// out = sum_gp N . val_e, divided by ipmax for the density call.
//
// On the uniform voxel box every element has the same 8 x 8 matrix, so the
// assembled K is a 27-point node stencil whose coefficients depend only on
// which of the node's 8 neighbouring elements exist: 3 x 3 x 3 node classes
// (lower face, interior, upper face per axis).  The table of 27 classes x 27
// neighbour slots is assembled once on the host in the reference's order
// (ascending element id) and the solve runs matrix-free: Ap = K p reads the
// class row from shared memory and p from a register window of 3 planes
// that marches along z.  The CG iteration
// reuses the device-resident scalar kernels of the elasticity solve (one
// stop-flag read per graph replay of `kHelmChunk` iterations).
#include <cmath>

#include "internal.cuh"

namespace icarat_b200
{

// the generic CG kernels of pcg.cu
__global__ void k_cg_init(int n, const double *__restrict__ b,
                          const double *__restrict__ invd, double *__restrict__ x,
                          double *__restrict__ r, double *__restrict__ z,
                          double *__restrict__ p, double *__restrict__ partials,
                          CgScalars *s, double tol, int maxit, int jacobi);
__global__ void k_cg_update_jacobi(int n, const double *__restrict__ invd,
                                   double *__restrict__ x, double *__restrict__ r,
                                   double *__restrict__ z,
                                   const double *__restrict__ p,
                                   const double *__restrict__ Ap,
                                   double *__restrict__ partials, CgScalars *s);
__global__ void k_cg_pupdate(int n, const double *__restrict__ z,
                             double *__restrict__ p, const CgScalars *s);

namespace
{

constexpr int kHelmChunk = 16;
constexpr int kHelmThreads = 256;
constexpr int kHelmClasses = 27;

struct HelmGrid
{
  int nx, ny, nz, NX, NY, numnp, nelx;
};

// integrals of the shape functions over the element: sum_gp N_a jac (the
// right-hand side weights) and sum_gp N_a (the readout weights); corners in
// bit order a = ax + 2 ay + 4 az
struct HelmWeights
{
  double nj[8], ns[8];
};

HelmGrid hgrid(const icarat_ctx *c)
{
  return HelmGrid{c->nx, c->ny, c->nz, c->NX, c->NY, c->numnp, c->nelx};
}

__device__ __forceinline__ int node_class(int i, int n)
{
  return i == 0 ? 0 : (i == n - 1 ? 2 : 1);
}

// F = sum over the node's elements of s_e nj[a] (/8 for the sensitivity
// call), elements in ascending id like the reference's assembly
__global__ void k_helm_rhs(HelmGrid g, HelmWeights w, const double *__restrict__ in,
                           double *__restrict__ F, int sens)
{
  for(int n = blockIdx.x * blockDim.x + threadIdx.x; n < g.numnp;
      n += gridDim.x * blockDim.x)
  {
    const int i = n % g.NX, rest = n / g.NX, j = rest % g.NY, k = rest / g.NY;
    double f = 0.0;
    for(int oz = -1; oz <= 0; oz++)
      for(int oy = -1; oy <= 0; oy++)
        for(int ox = -1; ox <= 0; ox++)
        {
          const int ei = i + ox, ej = j + oy, ek = k + oz;
          if(ei < 0 || ei >= g.nx || ej < 0 || ej >= g.ny || ek < 0 || ek >= g.nz)
            continue;
          const int a = -ox - 2 * oy - 4 * oz;
          double fe = __dmul_rn(__ldg(in + ei + (long)ej * g.nx + (long)ek * g.nx * g.ny),
                                w.nj[a]);
          if(sens)
            fe = __ddiv_rn(fe, 8.0);
          f = __dadd_rn(f, fe);
        }
    F[n] = f;
  }
}

// inverse of the stencil's centre coefficient (the Jacobi preconditioner)
__global__ void k_helm_invd(HelmGrid g, const double *__restrict__ coef,
                            double *__restrict__ invd)
{
  for(int n = blockIdx.x * blockDim.x + threadIdx.x; n < g.numnp;
      n += gridDim.x * blockDim.x)
  {
    const int i = n % g.NX, rest = n / g.NX, j = rest % g.NY, k = rest / g.NY;
    const int NZ = g.nz + 1;
    const int cls = node_class(i, g.NX) + 3 * node_class(j, g.NY) + 9 * node_class(k, NZ);
    invd[n] = 1.0 / coef[27 * cls + 13];
  }
}

// Ap = K p and alpha = zr / (p . Ap).
//
// A block of 32 x 8 threads owns a tile of 32 x 8 node columns and marches
// through kHelmTz planes of it: each thread keeps p of its 3 x 3 neighbour
// columns on planes k-1, k, k+1 in registers and loads one new plane (9
// values) per node instead of 27.  Neighbour slot q = (dk+1) 9 + (dj+1) 3 +
// (di+1) is also the window index; values outside the box are held as 0
// and their class coefficients are 0 (no element reaches them), so no read
// leaves the box.
constexpr int kHelmTx = 32, kHelmTy = 8, kHelmTz = 16;

__device__ __forceinline__ void helm_load_plane(double (&d)[9], const double *__restrict__ col,
                                                int k, int NZ, long plane, int NX, bool xm,
                                                bool xp, bool ym, bool yp)
{
  const bool in = k >= 0 && k < NZ;
  const double *q = col + (long)k * plane;
#pragma unroll
  for(int dy = -1; dy <= 1; dy++)
#pragma unroll
    for(int dx = -1; dx <= 1; dx++)
    {
      const bool ok = in && (dx >= 0 || xm) && (dx <= 0 || xp) && (dy >= 0 || ym) &&
                      (dy <= 0 || yp);
      d[(dy + 1) * 3 + dx + 1] = ok ? __ldg(q + dx + (long)dy * NX) : 0.0;
    }
}

__global__ void __launch_bounds__(kHelmTx * kHelmTy)
    k_helm_spmv(HelmGrid g, const double *__restrict__ coef, const double *__restrict__ p,
                double *__restrict__ Ap, double *__restrict__ partials, CgScalars *s)
{
  __shared__ double cs[kHelmClasses * 27];
  __shared__ double sh[64];
  if(s->done)
    return;
  for(int t = threadIdx.x; t < kHelmClasses * 27; t += blockDim.x)
    cs[t] = coef[t];
  __syncthreads();
  const int NZ = g.nz + 1;
  const long plane = (long)g.NX * g.NY;
  const int tiles_x = (g.NX + kHelmTx - 1) / kHelmTx, tiles_y = (g.NY + kHelmTy - 1) / kHelmTy;
  const int tiles = tiles_x * tiles_y * ((NZ + kHelmTz - 1) / kHelmTz);
  double dot = 0.0;
  for(int t = blockIdx.x; t < tiles; t += gridDim.x)
  {
    const int i = (t % tiles_x) * kHelmTx + (threadIdx.x & 31);
    const int j = (t / tiles_x % tiles_y) * kHelmTy + (threadIdx.x >> 5);
    const int k0 = t / (tiles_x * tiles_y) * kHelmTz;
    const int k1 = min(k0 + kHelmTz, NZ);
    if(i >= g.NX || j >= g.NY)
      continue;
    const bool xm = i > 0, xp = i < g.NX - 1, ym = j > 0, yp = j < g.NY - 1;
    const int cxy = node_class(i, g.NX) + 3 * node_class(j, g.NY);
    const long c0 = i + (long)j * g.NX;
    const double *col = p + c0;
    double w0[9], w1[9], w2[9];
    helm_load_plane(w0, col, k0 - 1, NZ, plane, g.NX, xm, xp, ym, yp);
    helm_load_plane(w1, col, k0, NZ, plane, g.NX, xm, xp, ym, yp);
    for(int k = k0; k < k1; k++)
    {
      helm_load_plane(w2, col, k + 1, NZ, plane, g.NX, xm, xp, ym, yp);
      const double *cf = cs + 27 * (cxy + 9 * node_class(k, NZ));
      double acc = 0.0;
#pragma unroll
      for(int q = 0; q < 9; q++)
        acc += cf[q] * w0[q];
#pragma unroll
      for(int q = 0; q < 9; q++)
        acc += cf[9 + q] * w1[q];
#pragma unroll
      for(int q = 0; q < 9; q++)
        acc += cf[18 + q] * w2[q];
      Ap[c0 + k * plane] = acc;
      dot += w1[4] * acc;
#pragma unroll
      for(int q = 0; q < 9; q++)
      {
        w0[q] = w1[q];
        w1[q] = w2[q];
      }
    }
  }
  double v[1] = {dot};
  block_sum<1>(v, sh);
  if(threadIdx.x == 0)
    partials[blockIdx.x] = v[0];
  if(last_block(&s->counter))
  {
    double t[1];
    sum_partials<1>(partials, gridDim.x, t, sh);
    if(threadIdx.x == 0)
    {
      s->pAp = t[0];
      s->alpha = s->zr / t[0];
      s->counter = 0;
    }
  }
}

// out_e = sum_a ns[a] val[node_a] (/8 for the density call)
__global__ void k_helm_out(HelmGrid g, HelmWeights w, const double *__restrict__ val,
                           double *__restrict__ out, int sens)
{
  const long plane = (long)g.NX * g.NY;
  for(int e = blockIdx.x * blockDim.x + threadIdx.x; e < g.nelx;
      e += gridDim.x * blockDim.x)
  {
    const int i = e % g.nx, j = (e / g.nx) % g.ny, k = e / (g.nx * g.ny);
    const long n0 = i + (long)j * g.NX + k * plane;
    double s = 0.0;
#pragma unroll
    for(int a = 0; a < 8; a++)
    {
      const long m = n0 + (a & 1) + ((a >> 1) & 1) * (long)g.NX + ((a >> 2) & 1) * plane;
      s = __dadd_rn(s, __dmul_rn(w.ns[a], __ldg(val + m)));
    }
    out[e] = sens ? s : __ddiv_rn(s, 8.0);
  }
}

int blocks_for(long n, int threads, int cap)
{
  long b = (n + threads - 1) / threads;
  if(b > cap)
    b = cap;
  return b < 1 ? 1 : (int)b;
}

} // namespace

// The 8 x 8 element matrix of one hx x hy x hz voxel and its shape-function
// integrals, 2 x 2 x 2 Gauss points (makeKeFint, filter_helm.hpp:203-217).
// The voxel's Jacobian is diag(hx, hy, hz) / 2.
void helm_element(double hx, double hy, double hz, double R, double *ke, double *nj,
                  double *ns)
{
  const double g = 1.0 / std::sqrt(3.0);
  const double cdiff = std::pow(R / (2.0 * std::sqrt(3.0)), 2);
  const double h[3] = {hx, hy, hz};
  const double jac = (hx * 0.5) * (hy * 0.5) * (hz * 0.5);
  for(int t = 0; t < 64; t++)
    ke[t] = 0.0;
  for(int a = 0; a < 8; a++)
    nj[a] = ns[a] = 0.0;
  for(int ip = 0; ip < 8; ip++)
  {
    const double r[3] = {(ip & 1) ? g : -g, (ip & 2) ? g : -g, (ip & 4) ? g : -g};
    double N[8], B[3][8];
    for(int a = 0; a < 8; a++)
    {
      double f[3], df[3];
      for(int d = 0; d < 3; d++)
      {
        const double sgn = ((a >> d) & 1) ? 1.0 : -1.0;
        f[d] = 1.0 + sgn * r[d];
        df[d] = sgn;
      }
      N[a] = 0.125 * f[0] * f[1] * f[2];
      B[0][a] = 0.125 * df[0] * f[1] * f[2] * (2.0 / h[0]);
      B[1][a] = 0.125 * f[0] * df[1] * f[2] * (2.0 / h[1]);
      B[2][a] = 0.125 * f[0] * f[1] * df[2] * (2.0 / h[2]);
    }
    for(int a = 0; a < 8; a++)
    {
      for(int b = 0; b < 8; b++)
      {
        double sb = 0.0;
        for(int d = 0; d < 3; d++)
          sb += B[d][a] * cdiff * B[d][b];
        ke[8 * a + b] += (N[a] * N[b] + sb) * jac;
      }
      nj[a] += N[a] * jac;
      ns[a] += N[a];
    }
  }
}

// 27 node classes x 27 neighbour slots: class (cx, cy, cz), c = 0 on the
// lower face, 1 inside, 2 on the upper face of an axis; the node's elements
// sit at offsets o in {-1, 0}^3 (o = -1 exists unless c = 0, o = 0 unless
// c = 2) and are summed in ascending element id like the assembly of
// setFromTriplets over the reference's element loop.
static void helm_class_table(const double *ke, double *coef)
{
  for(int cz = 0; cz < 3; cz++)
    for(int cy = 0; cy < 3; cy++)
      for(int cx = 0; cx < 3; cx++)
      {
        const int cls = cx + 3 * cy + 9 * cz;
        const int cc[3] = {cx, cy, cz};
        for(int q = 0; q < 27; q++)
        {
          const int dd[3] = {q % 3 - 1, q / 3 % 3 - 1, q / 9 - 1};
          double v = 0.0;
          for(int oz = -1; oz <= 0; oz++)
            for(int oy = -1; oy <= 0; oy++)
              for(int ox = -1; ox <= 0; ox++)
              {
                const int o[3] = {ox, oy, oz};
                bool ok = true;
                int a = 0, b = 0;
                for(int d = 0; d < 3; d++)
                {
                  if((o[d] == -1 && cc[d] == 0) || (o[d] == 0 && cc[d] == 2))
                    ok = false;
                  const int ad = -o[d], bd = ad + dd[d];
                  if(bd < 0 || bd > 1)
                    ok = false;
                  a |= ad << d;
                  b |= (bd & 1) << d;
                }
                if(ok)
                  v += ke[8 * a + b];
              }
          coef[27 * cls + q] = v;
        }
      }
}

void helm_free(icarat_ctx *c)
{
  HelmState &H = c->helm;
  if(H.exec)
    cudaGraphExecDestroy(H.exec);
  for(double *p : {H.d_coef, H.d_invd, H.d_F, H.d_val, H.d_r, H.d_z, H.d_p, H.d_Ap,
                   H.d_partials})
    dfree(p);
  dfree(H.d_cg);
  H = HelmState{};
}

void helm_setup(icarat_ctx *c, double R)
{
  IREQUIRE(R >= 0.0 && std::isfinite(R), ICARAT_ERR_ARG, "filter radius must be >= 0");
  helm_free(c);
  HelmState &H = c->helm;
  H.radius = R;
  helm_element(c->hx, c->hy, c->hz, R, H.ke, H.nj, H.ns);
  double coef[kHelmClasses * 27];
  helm_class_table(H.ke, coef);
  const size_t n = (size_t)c->numnp;
  H.d_coef = dalloc(kHelmClasses * 27);
  ICK(cudaMemcpy(H.d_coef, coef, sizeof(coef), cudaMemcpyHostToDevice));
  H.d_invd = dalloc(n);
  H.d_F = dalloc(n);
  H.d_val = dalloc(n);
  H.d_r = dalloc(n);
  H.d_z = dalloc(n);
  H.d_p = dalloc(n);
  H.d_Ap = dalloc(n);
  H.d_partials = dalloc((size_t)kMaxRedBlocks * 2);
  ICK(cudaMalloc(&H.d_cg, sizeof(CgScalars)));
  ICK(cudaMemsetAsync(H.d_cg, 0, sizeof(CgScalars), c->stream));
  note_launch();
  k_helm_invd<<<blocks_for(n, kHelmThreads, 4 * c->sm_count), kHelmThreads, 0, c->stream>>>(
      hgrid(c), H.d_coef, H.d_invd);
  ICK(cudaGetLastError());
}

static void helm_iteration(icarat_ctx *c)
{
  HelmState &H = c->helm;
  const int n = c->numnp;
  const long tiles = (long)((c->NX + kHelmTx - 1) / kHelmTx) *
                    ((c->NY + kHelmTy - 1) / kHelmTy) * ((c->NZ + kHelmTz - 1) / kHelmTz);
  note_launch(3);
  k_helm_spmv<<<blocks_for(tiles, 1, kMaxRedBlocks), kHelmTx * kHelmTy, 0, c->stream>>>(
      hgrid(c), H.d_coef, H.d_p, H.d_Ap, H.d_partials, H.d_cg);
  k_cg_update_jacobi<<<c->red_blocks, kRedThreads, 0, c->stream>>>(
      n, H.d_invd, H.d_val, H.d_r, H.d_z, H.d_p, H.d_Ap, H.d_partials, H.d_cg);
  k_cg_pupdate<<<c->red_blocks, kRedThreads, 0, c->stream>>>(n, H.d_z, H.d_p, H.d_cg);
  ICK(cudaGetLastError());
}

// densityFilter (filter_helm.hpp:75-138) of the device vector in (nelx) into
// out (nelx); rtol / maxit of the CG (<= 0: the reference's 1e-10 / 10000)
int helm_filter(icarat_ctx *c, const double *in, double *out, bool is_sens, double rtol,
                int maxit, icarat_solve_info *info)
{
  HelmState &H = c->helm;
  IREQUIRE(H.d_coef != nullptr, ICARAT_ERR_STATE, "Helmholtz filter not set up");
  IREQUIRE(std::isfinite(rtol), ICARAT_ERR_ARG, "rtol must be finite");
  if(rtol <= 0.0)
    rtol = 1.0e-10;
  if(maxit <= 0)
    maxit = 10000;
  const int n = c->numnp;
  const int eb = blocks_for(n, kHelmThreads, 4 * c->sm_count);
  HelmWeights w;
  for(int a = 0; a < 8; a++)
  {
    w.nj[a] = H.nj[a];
    w.ns[a] = H.ns[a];
  }
  note_launch(2);
  k_helm_rhs<<<eb, kHelmThreads, 0, c->stream>>>(hgrid(c), w, in, H.d_F, is_sens ? 1 : 0);
  ICK(cudaGetLastError());
  k_cg_init<<<c->red_blocks, kRedThreads, 0, c->stream>>>(n, H.d_F, H.d_invd, H.d_val,
                                                          H.d_r, H.d_z, H.d_p, H.d_partials,
                                                          H.d_cg, rtol, maxit, 1);
  ICK(cudaGetLastError());
  if(!H.exec)
  {
    cudaGraph_t graph;
    ICK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    set_capturing(true);
    try
    {
      for(int k = 0; k < kHelmChunk; k++)
        helm_iteration(c);
    }
    catch(...)
    {
      set_capturing(false);
      cudaStreamEndCapture(c->stream, &graph);
      throw;
    }
    set_capturing(false);
    ICK(cudaStreamEndCapture(c->stream, &graph));
    ICK(cudaGraphInstantiate(&H.exec, graph, 0));
    cudaGraphDestroy(graph);
  }
  const long max_chunks = ((long)maxit + 1 + kHelmChunk - 1) / kHelmChunk + 1;
  for(long ch = 0; ch < max_chunks; ch++)
  {
    ICK(cudaMemcpyAsync(c->h_cg, H.d_cg, sizeof(CgScalars), cudaMemcpyDeviceToHost,
                        c->stream));
    ICK(cudaStreamSynchronize(c->stream));
    if(c->h_cg->done)
      break;
    ICK(cudaGraphLaunch(H.exec, c->stream));
    note_launch(3 * kHelmChunk);
  }
  note_launch();
  k_helm_out<<<blocks_for(c->nelx, kHelmThreads, 4 * c->sm_count), kHelmThreads, 0,
               c->stream>>>(hgrid(c), w, H.d_val, out, is_sens ? 1 : 0);
  ICK(cudaGetLastError());
  ICK(cudaMemcpyAsync(c->h_cg, H.d_cg, sizeof(CgScalars), cudaMemcpyDeviceToHost,
                      c->stream));
  ICK(cudaStreamSynchronize(c->stream));
  const CgScalars &s = *c->h_cg;
  const int status = s.done ? s.status : ICARAT_WARN_MAXITER;
  if(info)
  {
    *info = icarat_solve_info{};
    info->iterations = s.iter;
    info->rel_residual = s.bnorm > 0 ? s.rnorm / s.bnorm : 0.0;
    info->status = status;
  }
  return status;
}

} // namespace icarat_b200
