// Preconditioned conjugate gradients with device-resident scalars.
//
// Semantics of Solvers::ScalingCG (src/analysis/solver/CG.cpp:56-99), the
// hand-written twin of the "Eigen_CG" solver the samples call
// (solvers.cpp:63-91): zero initial guess, z = M^-1 r, alpha = (z.r)/(p.Ap),
// beta = (z.r)_new/(z.r)_old, stop after the iteration whose ||r|| <
// rtol ||b|| or once iter > maxit.  A zero right-hand side returns u = 0 in 0
// iterations (Eigen's early exit).
//
// Every scalar (alpha, beta, norms, the stop flag) lives in device memory:
// the last block of each reduction kernel finishes the sum in a fixed order
// and applies the scalar logic, so an iteration never waits for the host.
// The host replays a CUDA graph of `chunk` iterations and reads the stop flag
// once per chunk; kernels of iterations past convergence return at entry.
#include <cmath>
#include <map>
#include <tuple>

#include "stencil.cuh"

namespace icarat_b200
{

// x = 0, r = b, z = invd r (Jacobi only), zr, bnorm.
__global__ void k_cg_init(int n, const double *__restrict__ b,
                          const double *__restrict__ invd, double *__restrict__ x,
                          double *__restrict__ r, double *__restrict__ z,
                          double *__restrict__ p, double *__restrict__ partials,
                          CgScalars *s, double tol, int maxit, int jacobi)
{
  chain_wait();
  __shared__ double sh[64];
  double zr = 0.0, bb = 0.0;
  for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
      i += gridDim.x * blockDim.x)
  {
    const double bi = b[i];
    x[i] = 0.0;
    r[i] = bi;
    if(jacobi)
    {
      const double zi = bi * invd[i];
      z[i] = zi;
      p[i] = zi;
      zr += zi * bi;
    }
    bb += bi * bi;
  }
  double v[2] = {zr, bb};
  block_sum<2>(v, sh);
  if(threadIdx.x == 0)
  {
    partials[blockIdx.x] = v[0];
    partials[gridDim.x + blockIdx.x] = v[1];
  }
  if(last_block(&s->counter))
  {
    double t[2];
    sum_partials<2>(partials, gridDim.x, t, sh);
    if(threadIdx.x == 0)
    {
      s->zr = t[0];
      s->bnorm = sqrt(t[1]);
      s->rnorm = s->bnorm;
      s->tol = tol;
      s->maxit = maxit;
      s->iter = 0;
      s->status = ICARAT_OK;
      s->done = (t[1] == 0.0) ? 1 : 0;
      if(!(t[1] == t[1]))
      {
        s->done = 1;
        s->status = ICARAT_ERR_NAN;
      }
      s->counter = 0;
    }
  }
}

// Warm start from the solution x of a previous system (Ax = K x given):
// r = b - Ax, z = invd r (Jacobi only), zr, ||b|| and ||r||.  The stop test
// stays ||r|| < tol ||b||; a start that already meets it is done after 0
// iterations (Eigen's solveWithGuess checks the initial residual too).
__global__ void k_cg_init_warm(int n, const double *__restrict__ b,
                               const double *__restrict__ Ax,
                               const double *__restrict__ invd, double *__restrict__ r,
                               double *__restrict__ z, double *__restrict__ p,
                               double *__restrict__ partials, CgScalars *s, double tol,
                               int maxit, int jacobi)
{
  chain_wait();
  __shared__ double sh[96];
  double zr = 0.0, bb = 0.0, rr = 0.0;
  for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
      i += gridDim.x * blockDim.x)
  {
    const double bi = b[i];
    const double ri = bi - Ax[i];
    r[i] = ri;
    if(jacobi)
    {
      const double zi = ri * invd[i];
      z[i] = zi;
      p[i] = zi;
      zr += zi * ri;
    }
    bb += bi * bi;
    rr += ri * ri;
  }
  double v[3] = {zr, bb, rr};
  block_sum<3>(v, sh);
  if(threadIdx.x == 0)
  {
    partials[blockIdx.x] = v[0];
    partials[gridDim.x + blockIdx.x] = v[1];
    partials[2 * gridDim.x + blockIdx.x] = v[2];
  }
  if(last_block(&s->counter))
  {
    double t[3];
    sum_partials<3>(partials, gridDim.x, t, sh);
    if(threadIdx.x == 0)
    {
      s->zr = t[0];
      s->bnorm = sqrt(t[1]);
      s->rnorm = sqrt(t[2]);
      s->rr = t[2];
      s->tol = tol;
      s->maxit = maxit;
      s->iter = 0;
      s->status = ICARAT_OK;
      s->done = (t[1] == 0.0 || s->rnorm < tol * s->bnorm) ? 1 : 0;
      if(!(t[1] == t[1]) || !(t[2] == t[2]))
      {
        s->done = 1;
        s->status = ICARAT_ERR_NAN;
      }
      s->counter = 0;
    }
  }
}

// Ap = K p, alpha = zr / (p . Ap)
__global__ void __launch_bounds__(128)
    k_cg_spmv(GridDev g, MarchPlan m, KeParam ke, const double *__restrict__ E,
              const uint8_t *__restrict__ fix, const double *__restrict__ p,
              double *__restrict__ Ap, double *__restrict__ partials,
              CgScalars *s)
{
  chain_wait();
  __shared__ double sh[32];
  if(s->done)
    return;
  double dot = 0.0;
  for(long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < m.items;
      t += (long)gridDim.x * blockDim.x)
  {
    int i, j, k0, k1;
    if(!march_item(g, m, t, i, j, k0, k1))
      continue;
    column_Ku(g, ke, E, p, i, j, k0, k1,
              [&](int k, const double(&acc)[3], const double(&uc)[3])
              {
                const int n = i + j * g.NX + k * g.NX * g.NY;
                const unsigned f = fix[n];
                const double y0 = (f & 1u) ? 0.0 : acc[0];
                const double y1 = (f & 2u) ? 0.0 : acc[1];
                const double y2 = (f & 4u) ? 0.0 : acc[2];
                Ap[n] = y0;
                Ap[(long)g.numnp + n] = y1;
                Ap[2L * g.numnp + n] = y2;
                dot += uc[0] * y0 + uc[1] * y1 + uc[2] * y2;
              });
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


// Jacobi: x += alpha p, r -= alpha Ap, z = invd r; beta, ||r||, stop test.
__global__ void k_cg_update_jacobi(int n, const double *__restrict__ invd,
                                   double *__restrict__ x, double *__restrict__ r,
                                   double *__restrict__ z,
                                   const double *__restrict__ p,
                                   const double *__restrict__ Ap,
                                   double *__restrict__ partials, CgScalars *s)
{
  chain_wait();
  __shared__ double sh[64];
  if(s->done)
    return;
  const double alpha = s->alpha;
  double zr = 0.0, rr = 0.0;
  for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
      i += gridDim.x * blockDim.x)
  {
    x[i] += alpha * p[i];
    const double ri = r[i] - alpha * Ap[i];
    r[i] = ri;
    const double zi = ri * invd[i];
    z[i] = zi;
    zr += zi * ri;
    rr += ri * ri;
  }
  double v[2] = {zr, rr};
  block_sum<2>(v, sh);
  if(threadIdx.x == 0)
  {
    partials[blockIdx.x] = v[0];
    partials[gridDim.x + blockIdx.x] = v[1];
  }
  if(last_block(&s->counter))
  {
    double t[2];
    sum_partials<2>(partials, gridDim.x, t, sh);
    if(threadIdx.x == 0)
    {
      s->zr_new = t[0];
      s->beta = t[0] / s->zr;
      s->zr = t[0];
      cg_check(s, t[1]);
      s->counter = 0;
    }
  }
}

// MG: x += alpha p, r -= alpha Ap; ||r||, stop test (z comes from a V-cycle).
// With x0 set, also the V-cycle's first Chebyshev step on the finest level
// from zero (k_cheb_first fused): d0 = x0 = inv_theta invd0 r.
__global__ void k_cg_update_r(int n, double *__restrict__ x,
                              double *__restrict__ r,
                              const double *__restrict__ p,
                              const double *__restrict__ Ap,
                              double *__restrict__ partials, CgScalars *s,
                              const double *__restrict__ invd0, double inv_theta,
                              double *__restrict__ x0, double *__restrict__ d0)
{
  chain_wait();
  __shared__ double sh[32];
  if(s->done)
    return;
  const double alpha = s->alpha;
  double rr = 0.0;
  for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
      i += gridDim.x * blockDim.x)
  {
    x[i] += alpha * p[i];
    const double ri = r[i] - alpha * Ap[i];
    r[i] = ri;
    rr += ri * ri;
    if(x0)
    {
      const double di = inv_theta * invd0[i] * ri;
      d0[i] = di;
      x0[i] = di;
    }
  }
  double v[1] = {rr};
  block_sum<1>(v, sh);
  if(threadIdx.x == 0)
    partials[blockIdx.x] = v[0];
  if(last_block(&s->counter))
  {
    double t[1];
    sum_partials<1>(partials, gridDim.x, t, sh);
    if(threadIdx.x == 0)
    {
      cg_check(s, t[0]);
      s->counter = 0;
    }
  }
}

// zr_new = z . r; beta = zr_new / zr (first = 1: p = z, no beta)
__global__ void k_cg_zr(int n, const double *__restrict__ z,
                        const double *__restrict__ r, double *__restrict__ partials,
                        CgScalars *s, int first)
{
  chain_wait();
  __shared__ double sh[32];
  if(s->done)
    return;
  double zr = 0.0;
  for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
      i += gridDim.x * blockDim.x)
    zr += z[i] * r[i];
  double v[1] = {zr};
  block_sum<1>(v, sh);
  if(threadIdx.x == 0)
    partials[blockIdx.x] = v[0];
  if(last_block(&s->counter))
  {
    double t[1];
    sum_partials<1>(partials, gridDim.x, t, sh);
    if(threadIdx.x == 0)
    {
      s->zr_new = t[0];
      s->beta = first ? 0.0 : t[0] / s->zr;
      s->zr = t[0];
      s->counter = 0;
    }
  }
}

// p = z + beta p   (CG.cpp:93: pk = beta * pk + Mrk)
__global__ void k_cg_pupdate(int n, const double *__restrict__ z,
                             double *__restrict__ p, const CgScalars *s)
{
  chain_wait();
  if(s->done)
    return;
  const double beta = s->beta;
  for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
      i += gridDim.x * blockDim.x)
    p[i] = beta * p[i] + z[i];
}

static GridDev fine_grid(const icarat_ctx *c)
{
  return GridDev{c->nx, c->ny, c->nz, c->NX, c->NY, c->NZ, c->numnp, c->nelx};
}

// column-march plan and block count of k_cg_spmv (blocks capped at the
// reduction's partial count; the kernel strides over the rest)
MarchPlan spmv_plan(const icarat_ctx *c, const GridDev &g, int &blocks)
{
  const MarchPlan m = march_launch(g, (const void *)k_cg_spmv, 128, c->sm_count, blocks);
  if(blocks > kMaxRedBlocks)
    blocks = kMaxRedBlocks;
  return m;
}

// One CG iteration (enqueued on c->stream).
static void enqueue_iteration(icarat_ctx *c, int method, int smooth,
                              const double *b, double *x)
{
  (void)b;
  const GridDev g = fine_grid(c);
  const int n = c->neq;
  const double *z = c->d_z;
  if(use_dmma(c, g))
  {
    DmArgs a;
    a.g = g;
    a.E = c->d_E;
    a.fix = c->d_fix;
    a.u = c->d_p;
    a.y = c->d_Ap;
    a.partials = c->d_partials;
    a.s = c->d_cg;
    launch_ku_dmma(c, TC_DOT, a, c->stream);
  }
  else
  {
    int blocks;
    const MarchPlan m = spmv_plan(c, g, blocks);
    note_launch();
    launch_chained(k_cg_spmv, blocks, 128, 0, c->stream, g, m, c->ke0, c->d_E, c->d_fix,
                   c->d_p, c->d_Ap, c->d_partials, c->d_cg);
  }
  if(method == ICARAT_SOLVER_JACOBI_PCG)
  {
    note_launch();
    launch_chained(k_cg_update_jacobi, c->red_blocks, kRedThreads, 0, c->stream, n,
                   c->d_invd, x, c->d_r, c->d_z, c->d_p, c->d_Ap, c->d_partials, c->d_cg);
  }
  else
  {
    note_launch();
    // the update also takes the finest level's first smoothing step
    MgLevel &L0 = c->mg[0];
    const double lm = c->lam_max_dk, theta = 0.5 * (lm + 0.1 * lm);
    launch_chained(k_cg_update_r, c->red_blocks, kRedThreads, 0, c->stream, n, x, c->d_r,
                   c->d_p, c->d_Ap, c->d_partials, c->d_cg, L0.invd, 1.0 / theta, L0.x, L0.r);
    // z stays in the finest level's x (overwritten only by the next
    // iteration's update, after z . r and the p update have read it)
    mg_vcycle(c, c->d_r, nullptr, smooth, true);
    z = c->mg[0].x;
    note_launch();
    launch_chained(k_cg_zr, c->red_blocks, kRedThreads, 0, c->stream, n, z, c->d_r,
                   c->d_partials, c->d_cg, 0);
  }
  note_launch();
  launch_chained(k_cg_pupdate, c->red_blocks, kRedThreads, 0, c->stream, n, z, c->d_p,
                 c->d_cg);
}

void release_graphs(icarat_ctx *c)
{
  for(auto &kv : c->graphs)
    cudaGraphExecDestroy(kv.second);
  c->graphs.clear();
}

int solve_full(icarat_ctx *c, const icarat_solve_opts *o, const double *d_b,
               double *d_x, icarat_solve_info *info)
{
  IREQUIRE(c->design_set, ICARAT_ERR_STATE, "set the design before solving");
  if(o->method == ICARAT_SOLVER_MIXED_IR || o->method == ICARAT_SOLVER_LEARNED_FPCG)
    return mixed_solve(c, o, d_b, d_x, info);
  const int method = o->method;
  IREQUIRE(method == ICARAT_SOLVER_JACOBI_PCG || method == ICARAT_SOLVER_MG_PCG,
           ICARAT_ERR_ARG, "unknown solver method");
  // the V-cycles of this solve stop with it (the iterations a graph chunk
  // holds past convergence launch, find the flag set and return)
  HaltScope halt(c, method == ICARAT_SOLVER_MG_PCG ? &c->d_cg->done : nullptr);
  const GridDev g = fine_grid(c);
  const int n = c->neq;
  IREQUIRE(o->fp64_tc >= -1 && o->fp64_tc <= 1, ICARAT_ERR_ARG, "fp64_tc must be -1, 0 or 1");
  c->fp64_tc = o->fp64_tc;
  int levels = 0, smooth = 0;
  if(method == ICARAT_SOLVER_MG_PCG)
  {
    levels = o->mg_levels > 0 ? o->mg_levels : 4;
    smooth = o->mg_smooth > 0 ? o->mg_smooth : 2;
    IREQUIRE(o->coarse_op == ICARAT_COARSE_REDISCRETISED || o->coarse_op == ICARAT_COARSE_GALERKIN,
             ICARAT_ERR_ARG, "coarse_op must be ICARAT_COARSE_REDISCRETISED or _GALERKIN");
    c->mg_galerkin_req = o->coarse_op == ICARAT_COARSE_GALERKIN ? 1 : 0;
    mg_setup(c, levels, o->coarse_lag != 0);
  }
  else
    launch_diag(c, g, c->d_E, c->d_fix, c->d_invd);
  int chunk = o->chunk > 0 ? o->chunk : (method == ICARAT_SOLVER_MG_PCG ? 4 : 16);

  // warm start: the context's own solution buffer holds a previous solution
  const bool warm = o->warm_start != 0 && c->have_u && d_x == c->d_u;
  if(warm)
  {
    launch_apply_K(c, g, c->d_E, c->d_fix, d_x, c->d_Ap, nullptr);
    note_launch();
    k_cg_init_warm<<<c->red_blocks, kRedThreads, 0, c->stream>>>(
        n, d_b, c->d_Ap, c->d_invd, c->d_r, c->d_z, c->d_p, c->d_partials, c->d_cg, o->rtol,
        o->maxit, method == ICARAT_SOLVER_JACOBI_PCG ? 1 : 0);
  }
  else
  {
    note_launch();
    k_cg_init<<<c->red_blocks, kRedThreads, 0, c->stream>>>(
        n, d_b, c->d_invd, d_x, c->d_r, c->d_z, c->d_p, c->d_partials, c->d_cg,
        o->rtol, o->maxit, method == ICARAT_SOLVER_JACOBI_PCG ? 1 : 0);
  }
  ICK(cudaGetLastError());
  if(method == ICARAT_SOLVER_MG_PCG)
  {
    // z0 = M r0, zr, p = z
    mg_vcycle(c, c->d_r, c->d_z, smooth);
    note_launch();
    k_cg_zr<<<c->red_blocks, kRedThreads, 0, c->stream>>>(n, c->d_z, c->d_r,
                                                          c->d_partials, c->d_cg, 1);
    ICK(cudaMemcpyAsync(c->d_p, c->d_z, sizeof(double) * n,
                        cudaMemcpyDeviceToDevice, c->stream));
  }
  const auto key =
      std::make_tuple(method + 4096 * (c->fp64_tc + 1), levels + 32 * c->coarse.cur, smooth,
                      chunk, (const void *)d_x);
  auto it = c->graphs.find(key);
  cudaGraphExec_t exec = nullptr;
  if(it == c->graphs.end())
  {
    cudaGraph_t graph;
    ICK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    set_capturing(true);
    try
    {
      for(int k = 0; k < chunk; k++)
        enqueue_iteration(c, method, smooth, d_b, d_x);
    }
    catch(...)
    {
      set_capturing(false);
      cudaStreamEndCapture(c->stream, &graph);
      throw;
    }
    set_capturing(false);
    ICK(cudaStreamEndCapture(c->stream, &graph));
    // kernel nodes per replay, for the launch counter
    size_t nn = 0;
    ICK(cudaGraphGetNodes(graph, nullptr, &nn));
    std::vector<cudaGraphNode_t> nodes(nn);
    ICK(cudaGraphGetNodes(graph, nodes.data(), &nn));
    int kernels = 0;
    for(auto nd : nodes)
    {
      cudaGraphNodeType t;
      ICK(cudaGraphNodeGetType(nd, &t));
      kernels += (t == cudaGraphNodeTypeKernel) ? 1 : 0;
    }
    ICK(cudaGraphInstantiate(&exec, graph, 0));
    cudaGraphDestroy(graph);
    c->graphs[key] = exec;
    c->graph_kernels[key] = kernels;
  }
  else
    exec = it->second;
  const int graph_kernels = c->graph_kernels[key];
  // iterations: cap + 1 like the reference loop, rounded up to whole chunks
  const long max_chunks = (long)(o->maxit + 1 + chunk - 1) / chunk + 1;
  for(long ch = 0; ch < max_chunks; ch++)
  {
    ICK(cudaMemcpyAsync(c->h_cg, c->d_cg, sizeof(CgScalars),
                        cudaMemcpyDeviceToHost, c->stream));
    ICK(cudaStreamSynchronize(c->stream));
    if(c->h_cg->done)
      break;
    ICK(cudaGraphLaunch(exec, c->stream));
    note_launch(graph_kernels);
  }
  if(method == ICARAT_SOLVER_MG_PCG)
    mg_join(c);
  ICK(cudaMemcpyAsync(c->h_cg, c->d_cg, sizeof(CgScalars),
                      cudaMemcpyDeviceToHost, c->stream));
  ICK(cudaStreamSynchronize(c->stream));
  const CgScalars &s = *c->h_cg;
  info->iterations = s.iter;
  info->rel_residual = s.bnorm > 0 ? s.rnorm / s.bnorm : 0.0;
  info->status = s.done ? s.status : ICARAT_WARN_MAXITER;
  info->refreshes = 0;
  info->learned_iterations = 0;
  return info->status;
}

} // namespace icarat_b200
