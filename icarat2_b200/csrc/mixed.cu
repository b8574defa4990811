// Mixed-precision solve of K u = b (no reference counterpart; the reference
// solves in FP64 only).
//
// The Krylov iteration runs on FP32 vectors: K p with the FP32 copy of Ke0 and
// of the element moduli, and an FP32 multigrid V-cycle as the preconditioner.
// Every dot product is accumulated in FP64 and every scalar is FP64.  The
// solution is refined in FP64: the iteration accumulates a correction x32;
// once the FP32 recurrence residual has fallen by the factor `refresh` below
// the last FP64 residual (or below the stopping threshold, or at the
// iteration cap, or kRefreshEvery iterations after the last refresh) the
// correction is added to the FP64 solution x, x32 is
// cleared and the residual is recomputed as r = b - K x with the FP64
// operator.  Convergence is decided on that FP64 residual only:
// ||b - K x|| < rtol ||b||; three refreshes in a row that cut it by less than
// 10 % end the FP32 iteration; then, and after a breakdown (a non-finite
// scalar), FP64 MG-PCG on the same hierarchy finishes the solve, started
// from the FP32 solution where that is finite (ill-conditioned systems such
// as solid islands floating in a 1e-9 void), and its status is the
// solve's.  The search direction
// survives the refresh, so the refinement does not restart the Krylov space;
// beta is the flexible
// (Polak-Ribiere) form beta = -(z . K p) / (p . K p), which keeps
// consecutive directions K-orthogonal under the inexact FP32 preconditioner
// and across a refresh.
//
// Like the FP64 solvers, all scalars live in device memory and the host
// replays a CUDA graph of `chunk` iterations, reading the stop flag once per
// chunk.
#include <cmath>

#include "stencil.cuh"

namespace icarat_b200
{

// Warm start: x kept, x32 = 0, r32 = b - K x in FP64; ||b|| and ||r||.
__global__ void __launch_bounds__(128)
    k_mx_init_warm(GridDev g, KeParam ke, const double *__restrict__ E,
                   const uint8_t *__restrict__ fix, const double *__restrict__ b,
                   const double *__restrict__ x, float *__restrict__ x32,
                   float *__restrict__ r32, double *__restrict__ partials, MxScalars *s,
                   double tol, double delta, int maxit)
{
  __shared__ double sh[64];
  double bb = 0.0, rr = 0.0;
  for(int n = blockIdx.x * blockDim.x + threadIdx.x; n < g.numnp;
      n += gridDim.x * blockDim.x)
  {
    double acc[3], uc[3];
    node_Ku(g, ke, E, x, n, acc, uc);
    const unsigned f = fix[n];
#pragma unroll
    for(int q = 0; q < 3; q++)
    {
      const long id = (long)q * g.numnp + n;
      const double bi = b[id];
      const double r = ((f >> q) & 1u) ? 0.0 : bi - acc[q];
      x32[id] = 0.0f;
      r32[id] = (float)r;
      bb += bi * bi;
      rr += r * r;
    }
  }
  double v[2] = {bb, rr};
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
      s->bb = t[0];
      s->rr = s->rr_ref = s->rr_true = t[1];
      s->tol2 = tol * tol * t[0];
      s->delta2 = delta * delta;
      s->maxit = maxit;
      s->iter = 0;
      s->refresh = 0;
      s->final_ = 0;
      s->nrefresh = 0;
      s->last_refresh = 0;
      s->nstall = 0;
      s->status = ICARAT_OK;
      s->done = (t[0] == 0.0 || t[1] < s->tol2) ? 1 : 0;
      if(!(t[0] == t[0]) || !(t[1] == t[1]))
      {
        s->done = 1;
        s->status = ICARAT_ERR_NAN;
      }
      s->counter = 0;
    }
  }
}

// x = 0, x32 = 0, r32 = b, ||b||.
__global__ void k_mx_init(int n, const double *__restrict__ b, double *__restrict__ x,
                          float *__restrict__ x32, float *__restrict__ r32,
                          double *__restrict__ partials, MxScalars *s, double tol,
                          double delta, int maxit)
{
  __shared__ double sh[32];
  double bb = 0.0;
  for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
  {
    const double bi = b[i];
    x[i] = 0.0;
    x32[i] = 0.0f;
    r32[i] = (float)bi;
    bb += bi * bi;
  }
  double v[1] = {bb};
  block_sum<1>(v, sh);
  if(threadIdx.x == 0)
    partials[blockIdx.x] = v[0];
  if(last_block(&s->counter))
  {
    double t[1];
    sum_partials<1>(partials, gridDim.x, t, sh);
    if(threadIdx.x == 0)
    {
      s->bb = t[0];
      s->rr = s->rr_ref = s->rr_true = t[0];
      s->tol2 = tol * tol * t[0];
      s->delta2 = delta * delta;
      s->maxit = maxit;
      s->iter = 0;
      s->refresh = 0;
      s->final_ = 0;
      s->nrefresh = 0;
      s->last_refresh = 0;
      s->nstall = 0;
      s->status = ICARAT_OK;
      s->done = (t[0] == 0.0) ? 1 : 0;
      if(!(t[0] == t[0]))
      {
        s->done = 1;
        s->status = ICARAT_ERR_NAN;
      }
      s->counter = 0;
    }
  }
}

// Ap = K32 p (constrained rows 0); alpha = zr / (p . Ap).
__global__ void __launch_bounds__(128)
    k_mx_spmv(GridDev g, MarchPlan m, KeParamF ke, const float *__restrict__ E,
              const uint8_t *__restrict__ fix, const float *__restrict__ p,
              float *__restrict__ Ap, double *__restrict__ partials, MxScalars *s)
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
              [&](int k, const float(&acc)[3], const float(&uc)[3])
              {
                const int n = i + j * g.NX + k * g.NX * g.NY;
                const unsigned f = fix[n];
#pragma unroll
                for(int q = 0; q < 3; q++)
                {
                  const float y = ((f >> q) & 1u) ? 0.0f : acc[q];
                  Ap[(long)q * g.numnp + n] = y;
                  dot += (double)uc[q] * (double)y;
                }
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

// x32 += alpha p, r32 -= alpha Ap; decide whether an FP64 refresh is due.
__global__ void k_mx_update(int n, float *__restrict__ x32, float *__restrict__ r32,
                            const float *__restrict__ p, const float *__restrict__ Ap,
                            double *__restrict__ partials, MxScalars *s)
{
  chain_wait();
  __shared__ double sh[32];
  if(s->done)
    return;
  const float alpha = (float)s->alpha;
  double rr = 0.0;
  for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
  {
    x32[i] = fmaf(alpha, p[i], x32[i]);
    const float ri = fmaf(-alpha, Ap[i], r32[i]);
    r32[i] = ri;
    rr += (double)ri * (double)ri;
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
      const double r2 = t[0];
      s->iter += 1;
      s->rr = r2;
      if(!(r2 == r2) || !(s->alpha == s->alpha))
      {
        s->done = 1;
        s->status = ICARAT_ERR_NAN;
      }
      else
      {
        s->final_ = s->iter > s->maxit ? 1 : 0;
        s->refresh = (r2 < s->delta2 * s->rr_ref || r2 < s->tol2 || s->final_ ||
                      s->iter - s->last_refresh >= kRefreshEvery)
                         ? 1
                         : 0;
      }
      s->counter = 0;
    }
  }
}

// Refresh, part 1: x += x32, x32 = 0.
__global__ void k_mx_flush(int n, double *__restrict__ x, float *__restrict__ x32,
                           const MxScalars *s)
{
  chain_wait();
  if(s->done || !s->refresh)
    return;
  for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
  {
    x[i] += (double)x32[i];
    x32[i] = 0.0f;
  }
}

// Refresh, part 2: r = b - K x in FP64, r32 = (float) r, stop test on ||r||.
__global__ void __launch_bounds__(128)
    k_mx_residual(GridDev g, MarchPlan m, KeParam ke, const double *__restrict__ E,
                  const uint8_t *__restrict__ fix, const double *__restrict__ b,
                  const double *__restrict__ x, float *__restrict__ r32,
                  double *__restrict__ partials, MxScalars *s)
{
  chain_wait();
  __shared__ double sh[32];
  if(s->done || !s->refresh)
    return;
  double rr = 0.0;
  for(long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < m.items;
      t += (long)gridDim.x * blockDim.x)
  {
    int i, j, k0, k1;
    if(!march_item(g, m, t, i, j, k0, k1))
      continue;
    column_Ku(g, ke, E, x, i, j, k0, k1,
              [&](int k, const double(&acc)[3], const double(&)[3])
              {
                const int n = i + j * g.NX + k * g.NX * g.NY;
                const unsigned f = fix[n];
#pragma unroll
                for(int q = 0; q < 3; q++)
                {
                  const long id = (long)q * g.numnp + n;
                  const double r = ((f >> q) & 1u) ? 0.0 : b[id] - acc[q];
                  r32[id] = (float)r;
                  rr += r * r;
                }
              });
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
      const double r2 = t[0];
      s->nstall = r2 > 0.81 * s->rr_true ? s->nstall + 1 : 0;
      s->rr_true = s->rr_ref = s->rr = r2;
      s->nrefresh += 1;
      s->last_refresh = s->iter;
      s->refresh = 0;
      if(!(r2 == r2))
      {
        s->done = 1;
        s->status = ICARAT_ERR_NAN;
      }
      else if(r2 < s->tol2)
      {
        s->done = 1;
        s->status = ICARAT_OK;
      }
      else if(s->final_)
      {
        s->done = 1;
        s->status = ICARAT_WARN_MAXITER;
      }
      else if(s->nstall >= 3)
      {
        // the FP64 residual is at the accuracy this operator and design allow
        s->done = 1;
        s->status = ICARAT_WARN_STAGNATION;
      }
      s->counter = 0;
    }
  }
}

// zr = z . r and beta = -(z . Ap) / pAp (first: beta = 0).
__global__ void k_mx_zr(int n, const float *__restrict__ z, const float *__restrict__ r,
                        const float *__restrict__ Ap, double *__restrict__ partials,
                        MxScalars *s, int first)
{
  chain_wait();
  __shared__ double sh[64];
  if(s->done)
    return;
  double zr = 0.0, zap = 0.0;
  for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
  {
    const double zi = z[i];
    zr += zi * (double)r[i];
    if(!first)
      zap += zi * (double)Ap[i];
  }
  double v[2] = {zr, zap};
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
      s->beta = first ? 0.0 : -t[1] / s->pAp;
      s->counter = 0;
    }
  }
}

// p = z + beta p (first: p = z)
__global__ void k_mx_pupdate(int n, const float *__restrict__ z, float *__restrict__ p,
                             const MxScalars *s, int first)
{
  chain_wait();
  if(s->done)
    return;
  const float beta = (float)s->beta;
  for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    p[i] = first ? z[i] : fmaf(beta, p[i], z[i]);
}

static float *falloc(size_t n)
{
  void *p = nullptr;
  cudaError_t e = cudaMalloc(&p, (n ? n : 1) * sizeof(float));
  if(e != cudaSuccess)
    throw Error{ICARAT_ERR_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e)};
  return static_cast<float *>(p);
}

__global__ void k_scale_f64(int n, double a, double *__restrict__ x)
{
  for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    x[i] = a == 0.0 ? 0.0 : a * x[i];
}

void mixed_alloc(icarat_ctx *c)
{
  if(c->f_x)
    return;
  const size_t nv = (size_t)c->neq;
  c->f_x = falloc(nv);
  c->f_r = falloc(nv);
  c->f_z = falloc(nv);
  c->f_p = falloc(nv);
  c->f_Ap = falloc(nv);
  ICK(cudaMalloc(&c->d_mx, sizeof(MxScalars)));
  ICK(cudaMemset(c->d_mx, 0, sizeof(MxScalars)));
  ICK(cudaMallocHost(&c->h_mx, sizeof(MxScalars)));
}

void mixed_free(icarat_ctx *c)
{
  for(void *p : {(void *)c->f_x, (void *)c->f_r, (void *)c->f_z, (void *)c->f_p,
                 (void *)c->f_Ap, (void *)c->d_mx})
    dfree(p);
  if(c->h_mx)
    cudaFreeHost(c->h_mx);
  c->f_x = c->f_r = c->f_z = c->f_p = c->f_Ap = nullptr;
  c->d_mx = c->h_mx = nullptr;
}

__global__ void k_round_f32(long n, const double *__restrict__ in, float *__restrict__ out)
{
  for(long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
      i += (long)gridDim.x * blockDim.x)
    out[i] = (float)in[i];
}

__global__ void k_widen_f64(long n, const float *__restrict__ in, double *__restrict__ out)
{
  for(long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
      i += (long)gridDim.x * blockDim.x)
    out[i] = (double)in[i];
}

void round_f32(icarat_ctx *c, long n, const double *in, float *out)
{
  note_launch();
  k_round_f32<<<c->red_blocks, kRedThreads, 0, c->stream>>>(n, in, out);
  ICK(cudaGetLastError());
}

void widen_f64(icarat_ctx *c, long n, const float *in, double *out)
{
  note_launch();
  k_widen_f64<<<c->red_blocks, kRedThreads, 0, c->stream>>>(n, in, out);
  ICK(cudaGetLastError());
}

void apply_K_lowp(icarat_ctx *c, int op, const float *u, float *y)
{
  const GridDev g{c->nx, c->ny, c->nz, c->NX, c->NY, c->NZ, c->numnp, c->nelx};
  if(op == ICARAT_OP_FP32)
  {
    launch_apply_K_f32(c, g, c->d_E32, c->d_fix, u, y);
    return;
  }
  IREQUIRE(op == ICARAT_OP_TC_BF16X3 || op == ICARAT_OP_TC_BF16, ICARAT_ERR_ARG,
           "unknown operator");
  TcArgs a;
  a.g = g;
  a.E = c->d_E32;
  a.fix = c->d_fix;
  a.u = u;
  a.y = y;
  launch_ku_tc(c, TC_APPLY, op == ICARAT_OP_TC_BF16X3 ? 3 : 1, a, c->stream);
}

// Operators of the FP32 iterations unless the options name others.  The
// smoother tolerates even the ~1e-3 relative error of the single-product
// BF16 tensor-core operator (the preconditioner is applied inexactly anyway:
// 15 iterations to 1e-6 at 256 x 128 x 128 with BF16, BF16 hi/lo and FP32
// alike, BF16 the fastest); the Krylov product K p does not (an inexact K p
// costs many more iterations), so it stays on the FP32 CUDA-core stencil.
constexpr int kDefaultFineOp = ICARAT_OP_TC_BF16;
constexpr int kDefaultKrylovOp = ICARAT_OP_FP32;

static int spmv_blocks(const icarat_ctx *c)
{
  int b = (c->numnp + 127) / 128;
  return b > kMaxRedBlocks ? kMaxRedBlocks : (b < 1 ? 1 : b);
}

// z = M r32, zr, beta, p update
// z = M r (the FP32 V-cycle), z . r, beta and p = z + beta p
static void enqueue_precondition(icarat_ctx *c, int smooth, int first)
{
  const int n = c->neq;
  // z stays in the finest level's x32 (read by z . r and the p update
  // before the next V-cycle overwrites it)
  mg_vcycle_f32(c, c->f_r, nullptr, smooth);
  const float *z = c->mg[0].x32;
  note_launch(2);
  launch_chained(k_mx_zr, c->red_blocks, kRedThreads, 0, c->stream, n, z, c->f_r, c->f_Ap,
                 c->d_partials, c->d_mx, first);
  launch_chained(k_mx_pupdate, c->red_blocks, kRedThreads, 0, c->stream, n, z, c->f_p,
                 c->d_mx, first);
}

// K p, the updates of x32 and r, and the FP64 refresh when one is due
static void enqueue_krylov_step(icarat_ctx *c, int krylov_op, const double *b, double *x);

static void enqueue_iteration(icarat_ctx *c, int smooth, int krylov_op, const double *b,
                              double *x)
{
  enqueue_krylov_step(c, krylov_op, b, x);
  enqueue_precondition(c, smooth, 0);
}

static void enqueue_krylov_step(icarat_ctx *c, int krylov_op, const double *b, double *x)
{
  const MgLevel &L = c->mg[0];
  const int n = c->neq;
  if(krylov_op == ICARAT_OP_FP32)
  {
    int blocks;
    const MarchPlan m = march_launch(L.g, (const void *)k_mx_spmv, 128, c->sm_count, blocks);
    note_launch();
    launch_chained(k_mx_spmv, blocks < kMaxRedBlocks ? blocks : kMaxRedBlocks, 128, 0,
                   c->stream, L.g, m, c->ke0f, L.E32, L.fix, c->f_p, c->f_Ap, c->d_partials,
                   c->d_mx);
  }
  else
  {
    TcArgs a;
    a.g = L.g;
    a.E = L.E32;
    a.fix = L.fix;
    a.u = c->f_p;
    a.y = c->f_Ap;
    a.partials = c->d_partials;
    a.s = c->d_mx;
    launch_ku_tc(c, TC_DOT, krylov_op == ICARAT_OP_TC_BF16X3 ? 3 : 1, a, c->stream);
  }
  note_launch(3);
  launch_chained(k_mx_update, c->red_blocks, kRedThreads, 0, c->stream, n, c->f_x, c->f_r,
                 c->f_p, c->f_Ap, c->d_partials, c->d_mx);
  launch_chained(k_mx_flush, c->red_blocks, kRedThreads, 0, c->stream, n, x, c->f_x, c->d_mx);
  int rblocks;
  const MarchPlan rm =
      march_launch(L.g, (const void *)k_mx_residual, 128, c->sm_count, rblocks);
  launch_chained(k_mx_residual, rblocks < kMaxRedBlocks ? rblocks : kMaxRedBlocks, 128, 0,
                 c->stream, L.g, rm, c->ke0, c->d_E, L.fix, b, (const double *)x, c->f_r,
                 c->d_partials, c->d_mx);
}

static const MxScalars &read_scalars(icarat_ctx *c)
{
  ICK(cudaMemcpyAsync(c->h_mx, c->d_mx, sizeof(MxScalars), cudaMemcpyDeviceToHost, c->stream));
  ICK(cudaStreamSynchronize(c->stream));
  return *c->h_mx;
}

// iterations preconditioned by the net at most, before the multigrid takes over
constexpr int kLearnedMaxIterations = 50;

// Everything before the chunk loop: set-up, initial guess and residual, the
// first preconditioning (and the learned phase), and the captured iteration
// graph.  Asynchronous on the context's stream except for the learned phase.
void mixed_begin(icarat_ctx *c, const icarat_solve_opts *o, const double *d_b, double *d_x,
                 MixedRun &run)
{
  IREQUIRE(o->rtol >= 0.0, ICARAT_ERR_ARG, "rtol must be non-negative");
  IREQUIRE(o->refresh >= 0.0 && o->refresh < 1.0, ICARAT_ERR_ARG,
           "refresh must be in [0, 1)");
  const int levels = o->mg_levels > 0 ? o->mg_levels : 4;
  const int smooth = o->mg_smooth > 0 ? o->mg_smooth : 2;
  const double delta = o->refresh > 0.0 ? o->refresh : 1.0e-2;
  const int chunk = o->chunk > 0 ? o->chunk : 4;
  const int fine_op = o->fine_op > 0 ? o->fine_op : kDefaultFineOp;
  const int krylov_op = o->krylov_op > 0 ? o->krylov_op : kDefaultKrylovOp;
  for(int op : {fine_op, krylov_op})
    IREQUIRE(op == ICARAT_OP_FP32 || op == ICARAT_OP_TC_BF16X3 || op == ICARAT_OP_TC_BF16,
             ICARAT_ERR_ARG, "mixed solver operators must be FP32 or tensor-core");
  c->mx_fine_op = fine_op;
  const bool learned = o->method == ICARAT_SOLVER_LEARNED_FPCG;
  IREQUIRE(!learned || c->net, ICARAT_ERR_STATE,
           "attach a net with icarat_ctx_set_net before the learned solver");
  IREQUIRE(o->coarse_op == ICARAT_COARSE_REDISCRETISED || o->coarse_op == ICARAT_COARSE_GALERKIN,
           ICARAT_ERR_ARG, "coarse_op must be ICARAT_COARSE_REDISCRETISED or _GALERKIN");
  c->mg_galerkin_req = o->coarse_op == ICARAT_COARSE_GALERKIN ? 1 : 0;
  mg_setup(c, levels, o->coarse_lag != 0);
  mixed_alloc(c);
  // the V-cycles enqueued and captured here stop with the iteration
  HaltScope halt(c, &c->d_mx->done);
  const int n = c->neq;
  const double nfree = c->numeq > 0 ? (double)c->numeq : 1.0;
  if(learned)
  {
    // initial guess x0 = alpha s net(b / s), s = ||b|| over the free DOFs;
    // alpha = (x0 . b) / (x0 . K x0) (either sign) minimises the energy norm
    // of the error along x0, so the guess is never worse than 0 in that norm
    // (no finite alpha: start from 0)
    const double bb = device_dot(c, d_b, d_b, n);
    net_apply<double>(c->net, c, d_b, bb > 0.0 ? std::sqrt(bb) : 1.0, d_x);
    const GridDev g{c->nx, c->ny, c->nz, c->NX, c->NY, c->NZ, c->numnp, c->nelx};
    launch_apply_K(c, g, c->d_E, c->d_fix, d_x, c->d_Ap, nullptr);
    const double xb = device_dot(c, d_x, d_b, n), xkx = device_dot(c, d_x, c->d_Ap, n);
    double alpha = (xkx > 0.0 && std::isfinite(xkx) && std::isfinite(xb)) ? xb / xkx : 0.0;
    alpha = std::isfinite(alpha) ? alpha : 0.0;
    note_launch();
    k_scale_f64<<<c->red_blocks, kRedThreads, 0, c->stream>>>(n, alpha, d_x);
  }

  note_launch();
  if(o->warm_start || learned)
  {
    const MgLevel &L0 = c->mg[0];
    k_mx_init_warm<<<spmv_blocks(c), 128, 0, c->stream>>>(L0.g, c->ke0, c->d_E, L0.fix, d_b,
                                                          d_x, c->f_x, c->f_r, c->d_partials,
                                                          c->d_mx, o->rtol, delta, o->maxit);
  }
  else
    k_mx_init<<<c->red_blocks, kRedThreads, 0, c->stream>>>(
        n, d_b, d_x, c->f_x, c->f_r, c->d_partials, c->d_mx, o->rtol, delta, o->maxit);
  ICK(cudaGetLastError());
  int learned_its = 0;
  if(learned)
  {
    // the net preconditions while every iteration at least halves the
    // residual; the first iteration that does not is preconditioned by the
    // V-cycle, and so is every later one
    // z = net(r); usable only if z . r > 0 (checked before p is updated)
    // (the net is trained up to sign: z = -net(r) when net(r) . r < 0)
    auto net_precondition = [&](int first, double rr) -> bool
    {
      double s = rr > 0.0 ? std::sqrt(rr) : 1.0;
      for(int pass = 0; pass < 2; pass++)
      {
        net_apply<float>(c->net, c, c->f_r, s, c->f_z);
        note_launch();
        k_mx_zr<<<c->red_blocks, kRedThreads, 0, c->stream>>>(n, c->f_z, c->f_r, c->f_Ap,
                                                              c->d_partials, c->d_mx, first);
        const MxScalars &sz = read_scalars(c);
        if(!std::isfinite(sz.zr) || sz.zr == 0.0)
          return false;
        if(sz.zr > 0.0)
          break;
        s = -s;
      }
      if(!(c->h_mx->zr > 0.0))
        return false;
      note_launch();
      k_mx_pupdate<<<c->red_blocks, kRedThreads, 0, c->stream>>>(n, c->f_z, c->f_p, c->d_mx,
                                                                 first);
      return true;
    };
    const MxScalars &s0 = read_scalars(c);
    if(!s0.done)
    {
      double rr_prev = s0.rr_true;
      if(!net_precondition(1, rr_prev))
        enqueue_precondition(c, smooth, 1); // the net is unusable: multigrid only
      else
      {
        learned_its = 1;
        for(int k = 0; k < kLearnedMaxIterations; k++)
        {
          enqueue_krylov_step(c, krylov_op, d_b, d_x);
          const MxScalars &sk = read_scalars(c);
          if(sk.done)
            break;
          const double rr = sk.rr;
          if(!(rr <= 0.25 * rr_prev) || !net_precondition(0, rr))
          {
            enqueue_precondition(c, smooth, 0); // fallback to the multigrid V-cycle
            break;
          }
          learned_its++;
          rr_prev = rr;
        }
      }
    }
    net_check(c->net, c->stream);
  }
  else
    enqueue_precondition(c, smooth, 1);
  ICK(cudaGetLastError());

  // the operators are part of what a captured graph launches
  const auto key = std::make_tuple((int)ICARAT_SOLVER_MIXED_IR + 16 * fine_op + 256 * krylov_op,
                                   levels + 32 * c->coarse.cur, smooth, chunk,
                                   (const void *)d_x);
  auto it = c->graphs.find(key);
  cudaGraphExec_t exec = nullptr;
  if(it == c->graphs.end() || c->graph_b.count(key) == 0 || c->graph_b[key] != d_b)
  {
    if(it != c->graphs.end())
    {
      cudaGraphExecDestroy(it->second);
      c->graphs.erase(it);
    }
    cudaGraph_t graph;
    ICK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    set_capturing(true);
    try
    {
      for(int k = 0; k < chunk; k++)
        enqueue_iteration(c, smooth, krylov_op, d_b, d_x);
    }
    catch(...)
    {
      set_capturing(false);
      cudaStreamEndCapture(c->stream, &graph);
      throw;
    }
    set_capturing(false);
    ICK(cudaStreamEndCapture(c->stream, &graph));
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
    c->graph_b[key] = d_b;
  }
  else
    exec = it->second;
  run.exec = exec;
  run.kernels = c->graph_kernels[key];
  run.max_chunks = (long)(o->maxit + 1 + chunk - 1) / chunk + 1;
  run.chunks = 0;
  run.learned_its = learned_its;
  // the stop flag as it stands after the set-up (read by mixed_poll)
  ICK(cudaMemcpyAsync(c->h_mx, c->d_mx, sizeof(MxScalars), cudaMemcpyDeviceToHost,
                      c->stream));
}

// After the stream has passed the last copy of the scalars: true while the
// solve needs another chunk.
bool mixed_poll(icarat_ctx *c, const MixedRun &run)
{
  return !c->h_mx->done && run.chunks < run.max_chunks;
}

// One chunk of iterations (graph replay) and the copy of the scalars after it.
void mixed_chunk(icarat_ctx *c, MixedRun &run)
{
  ICK(cudaGraphLaunch(run.exec, c->stream));
  note_launch(run.kernels);
  run.chunks++;
  ICK(cudaMemcpyAsync(c->h_mx, c->d_mx, sizeof(MxScalars), cudaMemcpyDeviceToHost,
                      c->stream));
}

int mixed_finish(icarat_ctx *c, const MixedRun &run, icarat_solve_info *info)
{
  const MxScalars &s = *c->h_mx;
  info->iterations = s.iter;
  info->rel_residual = s.bb > 0 ? std::sqrt(s.rr_true / s.bb) : 0.0;
  info->status = s.done ? s.status : ICARAT_WARN_MAXITER;
  info->refreshes = s.nrefresh;
  info->learned_iterations = run.learned_its;
  return info->status;
}

int mixed_solve(icarat_ctx *c, const icarat_solve_opts *o, const double *d_b,
                double *d_x, icarat_solve_info *info)
{
  MixedRun run;
  mixed_begin(c, o, d_b, d_x, run);
  for(;;)
  {
    ICK(cudaStreamSynchronize(c->stream));
    if(!mixed_poll(c, run))
      break;
    mixed_chunk(c, run);
  }
  mg_join(c);
  ICK(cudaStreamSynchronize(c->stream));
  return mixed_fp64_finish(c, o, d_b, d_x, info, mixed_finish(c, run, info));
}

// FP64 finish: an FP32 iteration that stalled above the tolerance (or broke
// down) on an ill-conditioned system hands over to FP64 MG-PCG on the same
// hierarchy, started from its solution where that is finite.  st: the
// status of the FP32 iteration, info its result (updated).
int mixed_fp64_finish(icarat_ctx *c, const icarat_solve_opts *o, const double *d_b, double *d_x,
                      icarat_solve_info *info, int st)
{
  if(st == ICARAT_ERR_NAN || st == ICARAT_WARN_STAGNATION)
  {
    icarat_solve_opts f = *o;
    f.method = ICARAT_SOLVER_MG_PCG;
    f.chunk = 0;
    f.fp64_tc = 0;
    f.warm_start = st == ICARAT_WARN_STAGNATION ? 1 : 0;
    icarat_solve_info fi{};
    const int s2 = solve_full(c, &f, d_b, d_x, &fi);
    info->iterations += fi.iterations;
    info->rel_residual = fi.rel_residual;
    info->refreshes += fi.refreshes;
    info->status = s2;
    return s2;
  }
  return st;
}

} // namespace icarat_b200
