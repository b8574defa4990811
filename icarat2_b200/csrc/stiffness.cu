// Matrix-free FP64 stiffness operator on the voxel grid.
//
// Replaces LinearAnalysis::assemblingK and the sparse product inside the CG
// (src/analysis/linear.hpp:117-166, src/analysis/solver/CG.cpp:76-99).
// Work per node: 8 elements x 3 rows x 24 = 576 DFMA (1152 flop); compulsory
// bytes per node: 24 read + 24 written (+ 8 per element modulus).
#include "stencil.cuh"

namespace icarat_b200
{

// y = K u (constrained rows zeroed); optional per-block partial of u . y.
__global__ void __launch_bounds__(128)
    k_apply_K_f64(GridDev g, MarchPlan m, KeParam ke, const double *__restrict__ E,
                  const uint8_t *__restrict__ fix, const double *__restrict__ u,
                  double *__restrict__ y, double *__restrict__ partials)
{
  __shared__ double sh[32];
  double dot = 0.0;
  for(long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < m.items;
      t += (long)gridDim.x * blockDim.x)
  {
    int i, j, k0, k1;
    if(!march_item(g, m, t, i, j, k0, k1))
      continue;
    column_Ku(g, ke, E, u, i, j, k0, k1,
              [&](int k, const double(&acc)[3], const double(&uc)[3])
              {
                const int n = i + j * g.NX + k * g.NX * g.NY;
                const unsigned f = fix[n];
                const double y0 = (f & 1u) ? 0.0 : acc[0];
                const double y1 = (f & 2u) ? 0.0 : acc[1];
                const double y2 = (f & 4u) ? 0.0 : acc[2];
                y[n] = y0;
                y[(long)g.numnp + n] = y1;
                y[2L * g.numnp + n] = y2;
                dot += uc[0] * y0 + uc[1] * y1 + uc[2] * y2;
              });
  }
  if(partials)
  {
    double v[1] = {dot};
    block_sum<1>(v, sh);
    if(threadIdx.x == 0)
      partials[blockIdx.x] = v[0];
  }
}

// 1 / diag(K): d_(n,c) = sum_{e ∋ n} E_e Ke0[3a+c][3a+c]; 0 on constrained.
__global__ void k_inv_diag(GridDev g, KeParam ke, const double *__restrict__ E,
                           const uint8_t *__restrict__ fix,
                           double *__restrict__ invd)
{
  for(int n = blockIdx.x * blockDim.x + threadIdx.x; n < g.numnp;
      n += gridDim.x * blockDim.x)
  {
    const int i = n % g.NX;
    const int j = (n / g.NX) % g.NY;
    const int k = n / (g.NX * g.NY);
    double d[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for(int sz = 0; sz < 2; sz++)
#pragma unroll
      for(int sy = 0; sy < 2; sy++)
#pragma unroll
        for(int sx = 0; sx < 2; sx++)
        {
          const double e = load_E(E, g, i - 1 + sx, j - 1 + sy, k - 1 + sz);
          const int a = local_node(1 - sx, 1 - sy, 1 - sz);
#pragma unroll
          for(int c = 0; c < 3; c++)
            d[c] = fma(e, ke.k[(3 * a + c) * 25], d[c]);
        }
    const unsigned f = fix[n];
#pragma unroll
    for(int c = 0; c < 3; c++)
      // a zero diagonal is treated as 1, as Eigen's DiagonalPreconditioner
      // does for the "Eigen_CG" solver (solvers.cpp:63-91)
      invd[(long)c * g.numnp + n] = ((f >> c) & 1u) ? 0.0 : (d[c] != 0.0 ? 1.0 / d[c] : 1.0);
  }
}

// r = b - K x (constrained rows 0).  Used by multigrid.
__global__ void __launch_bounds__(128)
    k_residual_f64(GridDev g, KeParam ke, const double *__restrict__ E,
                   const uint8_t *__restrict__ fix, const double *__restrict__ b,
                   const double *__restrict__ x, double *__restrict__ r)
{
  for(int n = blockIdx.x * blockDim.x + threadIdx.x; n < g.numnp;
      n += gridDim.x * blockDim.x)
  {
    double acc[3], uc[3];
    node_Ku(g, ke, E, x, n, acc, uc);
    const unsigned f = fix[n];
#pragma unroll
    for(int c = 0; c < 3; c++)
      r[(long)c * g.numnp + n] = ((f >> c) & 1u) ? 0.0 : b[(long)c * g.numnp + n] - acc[c];
  }
}

// K u_D restricted to free rows: fint of the first assembly, whose element
// displacements are the prescribed values (linear.hpp:63-77 followed by
// elasticity.cpp:244-254).
__global__ void __launch_bounds__(128)
    k_fint_f64(GridDev g, KeParam ke, const double *__restrict__ E,
               const uint8_t *__restrict__ fix, const double *__restrict__ uD,
               double *__restrict__ y)
{
  for(int n = blockIdx.x * blockDim.x + threadIdx.x; n < g.numnp;
      n += gridDim.x * blockDim.x)
  {
    double acc[3], uc[3];
    node_Ku(g, ke, E, uD, n, acc, uc);
    const unsigned f = fix[n];
#pragma unroll
    for(int c = 0; c < 3; c++)
      y[(long)c * g.numnp + n] = ((f >> c) & 1u) ? 0.0 : acc[c];
  }
}

__global__ void k_dot(int n, const double *__restrict__ a,
                      const double *__restrict__ b, double *__restrict__ partials,
                      unsigned int *counter, double *__restrict__ result)
{
  __shared__ double sh[32];
  double s = 0.0;
  for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
      i += gridDim.x * blockDim.x)
    s = fma(a[i], b[i], s);
  double v[1] = {s};
  block_sum<1>(v, sh);
  if(threadIdx.x == 0)
    partials[blockIdx.x] = v[0];
  if(last_block(counter))
  {
    double t[1];
    sum_partials<1>(partials, gridDim.x, t, sh);
    if(threadIdx.x == 0)
    {
      *result = t[0];
      *counter = 0;
    }
  }
}

static int node_blocks(const GridDev &g, int threads)
{
  int b = (g.numnp + threads - 1) / threads;
  return b < 1 ? 1 : b;
}

// Below kDmmaMinNodes the element tiles would leave most SMs idle.  The
// column-march node stencil is the faster FP64 operator at every grid size
// measured on a B200 (35 us against 62 us at 129 x 65 x 65 nodes, 273 us
// against 331 us at 257 x 129 x 129), so the default (fp64_tc 0) is the
// stencil and the FP64 tensor cores run only when asked for.
constexpr int kDmmaMinNodes = 1 << 15;

bool use_dmma(const icarat_ctx *c, const GridDev &g)
{
  if(c->fp64_tc <= 0 || !dmma_fits(g))
    return false;
  return c->fp64_tc == 1 ? g.numnp >= kDmmaMinNodes : true;
}

void launch_apply_K(icarat_ctx *c, const GridDev &g, const double *E,
                    const uint8_t *fix, const double *u, double *y,
                    double *dot_partials)
{
  if(!dot_partials && use_dmma(c, g))
  {
    DmArgs a;
    a.g = g;
    a.E = E;
    a.fix = fix;
    a.u = u;
    a.y = y;
    launch_ku_dmma(c, TC_APPLY, a, c->stream);
    return;
  }
  int blocks;
  const MarchPlan m = march_launch(g, (const void *)k_apply_K_f64, 128, c->sm_count, blocks);
  if(dot_partials && blocks > kMaxRedBlocks)
    blocks = kMaxRedBlocks;
  note_launch();
  k_apply_K_f64<<<blocks, 128, 0, c->stream>>>(g, m, c->ke0, E, fix, u, y, dot_partials);
  ICK(cudaGetLastError());
}

// y = K u in FP32 (the FP32 copies of Ke0 and of the moduli)
__global__ void __launch_bounds__(128)
    k_apply_K_f32(GridDev g, MarchPlan m, KeParamF ke, const float *__restrict__ E,
                  const uint8_t *__restrict__ fix, const float *__restrict__ u,
                  float *__restrict__ y)
{
  for(long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < m.items;
      t += (long)gridDim.x * blockDim.x)
  {
    int i, j, k0, k1;
    if(!march_item(g, m, t, i, j, k0, k1))
      continue;
    column_Ku(g, ke, E, u, i, j, k0, k1,
              [&](int k, const float(&acc)[3], const float(&)[3])
              {
                const int n = i + j * g.NX + k * g.NX * g.NY;
                const unsigned f = fix[n];
#pragma unroll
                for(int c = 0; c < 3; c++)
                  y[(long)c * g.numnp + n] = ((f >> c) & 1u) ? 0.0f : acc[c];
              });
  }
}

void launch_apply_K_f32(icarat_ctx *c, const GridDev &g, const float *E,
                        const uint8_t *fix, const float *u, float *y)
{
  int blocks;
  const MarchPlan m = march_launch(g, (const void *)k_apply_K_f32, 128, c->sm_count, blocks);
  note_launch();
  k_apply_K_f32<<<blocks, 128, 0, c->stream>>>(g, m, c->ke0f, E, fix, u, y);
  ICK(cudaGetLastError());
}

void launch_diag(icarat_ctx *c, const GridDev &g, const double *E,
                 const uint8_t *fix, double *invd, cudaStream_t st)
{
  note_launch();
  k_inv_diag<<<node_blocks(g, 256), 256, 0, st ? st : c->stream>>>(g, c->ke0, E, fix, invd);
  ICK(cudaGetLastError());
}

void launch_residual(icarat_ctx *c, const GridDev &g, const double *E,
                     const uint8_t *fix, const double *b, const double *x,
                     double *r)
{
  note_launch();
  k_residual_f64<<<node_blocks(g, 128), 128, 0, c->stream>>>(g, c->ke0, E, fix,
                                                             b, x, r);
  ICK(cudaGetLastError());
}

void launch_fint(icarat_ctx *c, double *out)
{
  GridDev g{c->nx, c->ny, c->nz, c->NX, c->NY, c->NZ, c->numnp, c->nelx};
  note_launch();
  k_fint_f64<<<node_blocks(g, 128), 128, 0, c->stream>>>(g, c->ke0, c->d_E,
                                                         c->d_fix, c->d_uD, out);
  ICK(cudaGetLastError());
}

double device_dot(icarat_ctx *c, const double *a, const double *b, int n)
{
  note_launch();
  k_dot<<<c->red_blocks, kRedThreads, 0, c->stream>>>(
      n, a, b, c->d_partials, c->d_counter, c->d_scalar);
  ICK(cudaGetLastError());
  ICK(cudaMemcpyAsync(c->h_scalar, c->d_scalar, sizeof(double),
                      cudaMemcpyDeviceToHost, c->stream));
  ICK(cudaStreamSynchronize(c->stream));
  return c->h_scalar[0];
}

} // namespace icarat_b200
