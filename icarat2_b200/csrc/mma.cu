// Method of moving asymptotes (Svanberg), the MMASolver of
// src/optimization/opt-solver/MMASolver.cpp (after Aage / Dumas, MIT):
// Update (:66-82) = GenSub (:400-512), xold shift, then the dual
// interior-point method SolveDIP (:88-154).
//
// GenSub is one elementwise kernel that also writes block partials of the
// constraint constants b_j.  SolveDIP runs as one cooperative kernel: every
// Newton step needs, at the current dual point lambda, the sums
//   S_j = sum_i p_ij / (U_i - x_i) + q_ij / (x_i - L_i)         (DualGrad,
//         DualResidual)
//   H_jk = sum_i PQ_ij df2_i PQ_ik                               (DualHess)
// with x = x(lambda) of XYZofLAMBDA.  One pass over the elements produces both
// (the residual after a line search and the gradient / Hessian of the next
// step are taken at the same lambda), the grid synchronises once, and every
// block reduces the partials in the same order and performs the same m x m
// scalar work, so all blocks follow one identical trajectory.
#include <cooperative_groups.h>

#include <algorithm>
#include <cmath>

#include "internal.cuh"

namespace cg = cooperative_groups;

constexpr int kMmaMaxM = 8;

struct icarat_mma
{
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = true;
  int n = 0, m = 0, iter = 0;
  double xmamieps, epsimin, raa0, move, albefa, asyminit, asymdec, asyminc;
  double a[kMmaMaxM], c[kMmaMaxM], d[kMmaMaxM];
  double *low = nullptr, *upp = nullptr, *alpha = nullptr, *beta = nullptr,
         *p0 = nullptr, *q0 = nullptr, *pij = nullptr, *qij = nullptr,
         *xold1 = nullptr, *xold2 = nullptr;
  double *stage = nullptr;    // host-API staging
  double *partials = nullptr; // 2 x (m + m^2) x blocks  + m x blocks (b)
  int *loops = nullptr;       // [outer, newton]
  int *h_loops = nullptr;     // pinned
  int blocks = 0;
  int last_outer = 0, last_newton = 0;
};

namespace icarat_b200
{

struct MmaArgs
{
  int n, m, iter;
  double xmamieps, raa0, move, albefa, asyminit, asymdec, asyminc, epsimin;
  double a[kMmaMaxM], c[kMmaMaxM], gx[kMmaMaxM];
  double *x;
  const double *dfdx, *dgdx, *xmin, *xmax;
  double *low, *upp, *alpha, *beta, *p0, *q0, *pij, *qij;
  const double *xold1, *xold2;
  double *pb;   // b partials [m][blocks]
  double *pred; // 2 buffers of [(m + m^2)][blocks]
  int *loops;
};

// GenSub (MMASolver.cpp:400-512) + partials of b_j.
template <int M>
__global__ void __launch_bounds__(256) k_mma_gensub(MmaArgs A)
{
  __shared__ double sh[32 * (M > 0 ? M : 1)];
  double bpart[M > 0 ? M : 1];
#pragma unroll
  for(int j = 0; j < M; j++)
    bpart[j] = 0.0;
  for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < A.n;
      i += gridDim.x * blockDim.x)
  {
    const double xv = A.x[i], xmn = A.xmin[i], xmx = A.xmax[i];
    double lo, up;
    if(A.iter < 3)
    {
      lo = xv - A.asyminit * (xmx - xmn);
      up = xv + A.asyminit * (xmx - xmn);
    }
    else
    {
      const double x1 = A.xold1[i], x2 = A.xold2[i];
      const double zzz = (xv - x1) * (x1 - x2);
      const double gamma = zzz < 0.0 ? A.asymdec : (zzz > 0.0 ? A.asyminc : 1.0);
      lo = xv - gamma * (x1 - A.low[i]);
      up = xv + gamma * (A.upp[i] - x1);
      const double xmami = fmax(A.xmamieps, xmx - xmn);
      lo = fmax(lo, xv - 100.0 * xmami);
      lo = fmin(lo, xv - 1.0e-5 * xmami);
      up = fmax(up, xv + 1.0e-5 * xmami);
      up = fmin(up, xv + 100.0 * xmami);
      const double xmi = xmn - 1.0e-6, xma = xmx + 1.0e-6;
      if(xv < xmi)
      {
        lo = xv - (xma - xv) / 0.9;
        up = xv + (xma - xv) / 0.9;
      }
      if(xv > xma)
      {
        lo = xv - (xv - xmi) / 0.9;
        up = xv + (xv - xmi) / 0.9;
      }
    }
    A.low[i] = lo;
    A.upp[i] = up;
    double al = fmax(xmn, lo + A.albefa * (xv - lo));
    al = fmax(al, xv - A.move * (xmx - xmn));
    A.alpha[i] = fmin(al, xmx);
    double be = fmin(xmx, up - A.albefa * (up - xv));
    be = fmin(be, xv + A.move * (xmx - xmn));
    A.beta[i] = fmax(be, xmn);
    const double ux = up - xv, xl = xv - lo;
    const double ux2 = ux * ux, xl2 = xl * xl;
    const double xmamiinv = 1.0 / fmax(A.xmamieps, xmx - xmn);
    const double df = A.dfdx[i];
    const double pq = 0.001 * fabs(df) + A.raa0 * xmamiinv;
    A.p0[i] = ux2 * (fmax(0.0, df) + pq);
    A.q0[i] = xl2 * (fmax(0.0, -1.0 * df) + pq);
#pragma unroll
    for(int j = 0; j < M; j++)
    {
      const double gd = A.dgdx[(long)i * M + j];
      const double pqj = 0.001 * fabs(gd) + A.raa0 * xmamiinv;
      const double p = ux2 * (fmax(0.0, gd) + pqj);
      const double q = xl2 * (fmax(0.0, -1.0 * gd) + pqj);
      A.pij[(long)i * M + j] = p;
      A.qij[(long)i * M + j] = q;
      bpart[j] += p / ux + q / xl;
    }
  }
  if(M > 0)
  {
    block_sum<(M > 0 ? M : 1)>(bpart, sh);
    if(threadIdx.x == 0)
#pragma unroll
      for(int j = 0; j < M; j++)
        A.pb[j * gridDim.x + blockIdx.x] = bpart[j];
  }
}

// x(lambda) of XYZofLAMBDA for element i, plus the unclamped xp.
template <int M>
__device__ __forceinline__ void mma_x(const MmaArgs &A, int i, const double *lam,
                                      double &x, double &xp, double &pl, double &ql)
{
  pl = A.p0[i];
  ql = A.q0[i];
#pragma unroll
  for(int j = 0; j < M; j++)
  {
    pl += A.pij[(long)i * M + j] * lam[j];
    ql += A.qij[(long)i * M + j] * lam[j];
  }
  const double lo = A.low[i], up = A.upp[i];
  const double sp = sqrt(pl), sq = sqrt(ql);
  xp = (sp * lo + sq * up) / (sp + sq);
  x = xp;
  if(x < A.alpha[i])
    x = A.alpha[i];
  if(x > A.beta[i])
    x = A.beta[i];
}

// In-place LU without pivoting and the two sweeps (MMASolver.cpp:514-553).
template <int M>
__device__ void mma_lu_solve(double *K, double *x)
{
  for(int s = 0; s < M - 1; s++)
    for(int i = s + 1; i < M; i++)
    {
      K[i * M + s] = K[i * M + s] / K[s * M + s];
      for(int j = s + 1; j < M; j++)
        K[i * M + j] = K[i * M + j] - K[i * M + s] * K[s * M + j];
    }
  for(int i = 1; i < M; i++)
  {
    double a = 0.0;
    for(int j = 0; j < i; j++)
      a = a - K[i * M + j] * x[j];
    x[i] = x[i] + a;
  }
  x[M - 1] = x[M - 1] / K[(M - 1) * M + (M - 1)];
  for(int i = M - 2; i >= 0; i--)
  {
    double a = x[i];
    for(int j = i + 1; j < M; j++)
      a = a - K[i * M + j] * x[j];
    x[i] = a / K[i * M + i];
  }
}

template <int M> struct MmaShared
{
  double lam[M], mu[M], y[M], b[M], S[M], H[M * M], grad[M], hess[M * M],
      s[2 * M];
  double z, epsi, err;
  int go_outer, go_inner;
  double red[32 * (M + M * M)];
};

// One pass at the current lambda: S and H reduced grid-wide into sm.
template <int M>
__device__ void mma_pass(const MmaArgs &A, MmaShared<M> &sm, cg::grid_group &grid,
                         int buf)
{
  constexpr int NV = M + M * M;
  double acc[NV];
#pragma unroll
  for(int q = 0; q < NV; q++)
    acc[q] = 0.0;
  double lam[M];
#pragma unroll
  for(int j = 0; j < M; j++)
    lam[j] = sm.lam[j];
  for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < A.n;
      i += gridDim.x * blockDim.x)
  {
    double x, xp, pl, ql;
    mma_x<M>(A, i, lam, x, xp, pl, ql);
    const double ux = A.upp[i] - x, xl = x - A.low[i];
    // one reciprocal per distance, then products (the reference divides by
    // pow(., 3) and by each power separately; the values agree to rounding)
    const double rux = 1.0 / ux, rxl = 1.0 / xl;
    const double rux2 = rux * rux, rxl2 = rxl * rxl;
    double df2 = -1.0 / (2.0 * pl * (rux2 * rux) + 2.0 * ql * (rxl2 * rxl));
    if(xp < A.alpha[i])
      df2 = 0.0;
    if(xp > A.beta[i])
      df2 = 0.0;
    double PQ[M];
#pragma unroll
    for(int j = 0; j < M; j++)
    {
      const double p = A.pij[(long)i * M + j], q = A.qij[(long)i * M + j];
      acc[j] += p * rux + q * rxl;
      PQ[j] = p * rux2 - q * rxl2;
    }
#pragma unroll
    for(int j = 0; j < M; j++)
#pragma unroll
      for(int k = 0; k < M; k++)
        acc[M + j * M + k] += (PQ[j] * df2) * PQ[k];
  }
  block_sum<NV>(acc, sm.red);
  double *P = A.pred + (size_t)buf * NV * gridDim.x;
  if(threadIdx.x == 0)
#pragma unroll
    for(int q = 0; q < NV; q++)
      P[q * gridDim.x + blockIdx.x] = acc[q];
  grid.sync();
  double t[NV];
  sum_partials<NV>(P, gridDim.x, t, sm.red);
  if(threadIdx.x == 0)
  {
#pragma unroll
    for(int j = 0; j < M; j++)
      sm.S[j] = t[j];
#pragma unroll
    for(int q = 0; q < M * M; q++)
      sm.H[q] = t[M + q];
  }
  __syncthreads();
}

// XYZofLAMBDA scalar part: clamp lambda, y, z (MMASolver.cpp:362-373)
template <int M>
__device__ __forceinline__ void mma_yz(const MmaArgs &A, MmaShared<M> &sm)
{
  double lamai = 0.0;
  for(int j = 0; j < M; j++)
  {
    if(sm.lam[j] < 0.0)
      sm.lam[j] = 0;
    sm.y[j] = fmax(0.0, sm.lam[j] - A.c[j]);
    lamai += sm.lam[j] * A.a[j];
  }
  sm.z = fmax(0.0, 10.0 * (lamai - 1.0));
}

template <int M>
__global__ void __launch_bounds__(256) k_mma_dip(MmaArgs A)
{
  cg::grid_group grid = cg::this_grid();
  __shared__ MmaShared<M> sm;
  // b_j = -gx_j + sum_i (...)
  {
    double t[M];
    sum_partials<M>(A.pb, gridDim.x, t, sm.red);
    if(threadIdx.x == 0)
      for(int j = 0; j < M; j++)
        sm.b[j] = -A.gx[j] + t[j];
  }
  if(threadIdx.x == 0)
  {
    for(int j = 0; j < M; j++)
    {
      sm.lam[j] = A.c[j] / 2.0;
      sm.mu[j] = 1.0;
    }
    sm.epsi = 1.0;
    sm.err = 1.0;
    mma_yz<M>(A, sm);
  }
  __syncthreads();
  int buf = 0;
  mma_pass<M>(A, sm, grid, buf);
  buf ^= 1;
  int outloop = 0, newton = 0;
  while(sm.epsi > A.epsimin && outloop < 100)
  {
    outloop++;
    int loop = 0;
    while(sm.err > 0.9 * sm.epsi && loop < 100)
    {
      loop++;
      newton++;
      if(threadIdx.x == 0)
      {
        // gradient (DualGrad + the sign flip and barrier term, :112-116)
        for(int j = 0; j < M; j++)
        {
          const double gj = -sm.b[j] - A.a[j] * sm.z - sm.y[j] + sm.S[j];
          sm.grad[j] = -1.0 * gj - sm.epsi / sm.lam[j];
        }
        // DualHess scalar part (:297-339)
        for(int q = 0; q < M * M; q++)
          sm.hess[q] = sm.H[q];
        double lamai = 0.0;
        for(int j = 0; j < M; j++)
        {
          if(sm.lam[j] < 0.0)
            sm.lam[j] = 0.0;
          lamai += sm.lam[j] * A.a[j];
          if(sm.lam[j] > A.c[j])
            sm.hess[j * M + j] += -1.0;
          sm.hess[j * M + j] += -sm.mu[j] / sm.lam[j];
        }
        if(lamai > 0.0)
          for(int j = 0; j < M; j++)
            for(int k = 0; k < M; k++)
              sm.hess[j * M + k] += -10.0 * A.a[j] * A.a[k];
        double tr = 0.0;
        for(int j = 0; j < M; j++)
          tr += sm.hess[j * M + j];
        double corr = 1e-4 * tr / M;
        if(-1.0 * corr < 1.0e-7)
          corr = -1.0e-7;
        for(int j = 0; j < M; j++)
          sm.hess[j * M + j] += corr;
        // Newton direction
        if(M > 1)
        {
          mma_lu_solve<M>(sm.hess, sm.grad);
          for(int j = 0; j < M; j++)
            sm.s[j] = sm.grad[j];
        }
        else
          sm.s[0] = sm.grad[0] / sm.hess[0];
        for(int j = 0; j < M; j++)
          sm.s[M + j] = -sm.mu[j] + sm.epsi / sm.lam[j] - sm.s[j] * sm.mu[j] / sm.lam[j];
        // DualLineSearch (:214-236)
        double theta = 1.005;
        for(int j = 0; j < M; j++)
        {
          if(theta < -1.01 * sm.s[j] / sm.lam[j])
            theta = -1.01 * sm.s[j] / sm.lam[j];
          if(theta < -1.01 * sm.s[j + M] / sm.mu[j])
            theta = -1.01 * sm.s[j + M] / sm.mu[j];
        }
        theta = 1.0 / theta;
        for(int j = 0; j < M; j++)
        {
          sm.lam[j] = sm.lam[j] + theta * sm.s[j];
          sm.mu[j] = sm.mu[j] + theta * sm.s[j + M];
        }
        mma_yz<M>(A, sm);
      }
      __syncthreads();
      mma_pass<M>(A, sm, grid, buf);
      buf ^= 1;
      if(threadIdx.x == 0)
      {
        // DualResidual (:184-212)
        double nr = 0.0;
        for(int j = 0; j < M; j++)
        {
          const double r1 = -sm.b[j] - A.a[j] * sm.z - sm.y[j] + sm.mu[j] + sm.S[j];
          const double r2 = sm.mu[j] * sm.lam[j] - sm.epsi;
          if(nr < fabs(r1))
            nr = fabs(r1);
          if(nr < fabs(r2))
            nr = fabs(r2);
        }
        sm.err = nr;
      }
      __syncthreads();
    }
    if(threadIdx.x == 0)
      sm.epsi = sm.epsi * 0.1;
    __syncthreads();
  }
  // x = x(lambda) of the last XYZofLAMBDA
  double lam[M];
#pragma unroll
  for(int j = 0; j < M; j++)
    lam[j] = sm.lam[j];
  for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < A.n;
      i += gridDim.x * blockDim.x)
  {
    double x, xp, pl, ql;
    mma_x<M>(A, i, lam, x, xp, pl, ql);
    A.x[i] = x;
  }
  if(blockIdx.x == 0 && threadIdx.x == 0)
  {
    A.loops[0] = outloop;
    A.loops[1] = newton;
  }
}

template <int M> static void mma_launch(icarat_mma *h, MmaArgs &A)
{
  int per_sm = 0, sms = 0;
  ICK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_mma_dip<M>, 256, 0));
  ICK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->device));
  int blocks = sms * (per_sm > 1 ? 1 : per_sm);
  const int need = (h->n + 255) / 256;
  blocks = std::min(blocks, std::max(need, 1));
  IREQUIRE(blocks >= 1, ICARAT_ERR_CUDA, "no co-resident blocks for the MMA kernel");
  note_launch();
  k_mma_gensub<M><<<blocks, 256, 0, h->stream>>>(A);
  ICK(cudaGetLastError());
  // xold2 = xold1; xold1 = xval (MMASolver.cpp:73-75)
  ICK(cudaMemcpyAsync(h->xold2, h->xold1, sizeof(double) * h->n,
                      cudaMemcpyDeviceToDevice, h->stream));
  ICK(cudaMemcpyAsync(h->xold1, A.x, sizeof(double) * h->n, cudaMemcpyDeviceToDevice,
                      h->stream));
  void *args[] = {&A};
  note_launch();
  ICK(cudaLaunchCooperativeKernel((void *)k_mma_dip<M>, dim3(blocks), dim3(256), args,
                                  0, h->stream));
}

int mma_update_device(icarat_mma *h, double *x, const double *dfdx, const double *gx,
                      const double *dgdx, const double *xmin, const double *xmax)
{
  h->iter++;
  MmaArgs A;
  A.n = h->n;
  A.m = h->m;
  A.iter = h->iter;
  A.xmamieps = h->xmamieps;
  A.raa0 = h->raa0;
  A.move = h->move;
  A.albefa = h->albefa;
  A.asyminit = h->asyminit;
  A.asymdec = h->asymdec;
  A.asyminc = h->asyminc;
  A.epsimin = h->epsimin;
  for(int j = 0; j < kMmaMaxM; j++)
  {
    A.a[j] = j < h->m ? h->a[j] : 0.0;
    A.c[j] = j < h->m ? h->c[j] : 0.0;
    A.gx[j] = j < h->m ? gx[j] : 0.0;
  }
  A.x = x;
  A.dfdx = dfdx;
  A.dgdx = dgdx;
  A.xmin = xmin;
  A.xmax = xmax;
  A.low = h->low;
  A.upp = h->upp;
  A.alpha = h->alpha;
  A.beta = h->beta;
  A.p0 = h->p0;
  A.q0 = h->q0;
  A.pij = h->pij;
  A.qij = h->qij;
  A.xold1 = h->xold1;
  A.xold2 = h->xold2;
  A.pb = h->partials;
  A.pred = h->partials + (size_t)kMmaMaxM * 4096;
  A.loops = h->loops;
  switch(h->m)
  {
  case 1: mma_launch<1>(h, A); break;
  case 2: mma_launch<2>(h, A); break;
  case 3: mma_launch<3>(h, A); break;
  case 4: mma_launch<4>(h, A); break;
  case 5: mma_launch<5>(h, A); break;
  case 6: mma_launch<6>(h, A); break;
  case 7: mma_launch<7>(h, A); break;
  case 8: mma_launch<8>(h, A); break;
  default: throw Error{ICARAT_ERR_UNSUPPORTED, "MMA supports 1 <= m <= 8"};
  }
  ICK(cudaMemcpyAsync(h->h_loops, h->loops, 2 * sizeof(int), cudaMemcpyDeviceToHost,
                      h->stream));
  ICK(cudaStreamSynchronize(h->stream));
  h->last_outer = h->h_loops[0];
  h->last_newton = h->h_loops[1];
  return ICARAT_OK;
}

void mma_destroy(icarat_mma *h);

// stream: run on this stream (owned by the caller) or, when null, on a new one
void mma_create(int device, int n, int m, double a, double c, double d,
                icarat_mma **out, cudaStream_t stream)
{
  IREQUIRE(n >= 1 && m >= 1 && m <= kMmaMaxM, ICARAT_ERR_ARG,
           "MMA needs n >= 1 and 1 <= m <= 8");
  icarat_mma *h = new icarat_mma();
  try
  {
    h->device = device;
    ICK(cudaSetDevice(device));
    if(stream)
    {
      h->stream = stream;
      h->own_stream = false;
    }
    else
      ICK(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
    h->n = n;
    h->m = m;
    h->iter = 0;
    // MMASolver::MMASolver defaults (MMASolver.cpp:41-55)
    h->xmamieps = 1.0e-5;
    h->epsimin = std::sqrt((double)(n + m)) * 1e-9;
    h->raa0 = 0.00001;
    h->move = 0.15;
    h->albefa = 0.2;
    h->asyminit = 0.2;
    h->asymdec = 0.7;
    h->asyminc = 1.2;
    for(int j = 0; j < kMmaMaxM; j++)
    {
      h->a[j] = a;
      h->c[j] = c;
      h->d[j] = d;
    }
    for(double **p : {&h->low, &h->upp, &h->alpha, &h->beta, &h->p0, &h->q0,
                      &h->xold1, &h->xold2})
    {
      *p = dalloc(n);
      ICK(cudaMemset(*p, 0, sizeof(double) * n));
    }
    h->pij = dalloc((size_t)n * m);
    h->qij = dalloc((size_t)n * m);
    h->stage = dalloc((size_t)n * (4 + m) + kMmaMaxM);
    h->partials = dalloc((size_t)kMmaMaxM * 4096 +
                         2 * (size_t)(kMmaMaxM + kMmaMaxM * kMmaMaxM) * 4096);
    ICK(cudaMalloc(&h->loops, 2 * sizeof(int)));
    ICK(cudaMallocHost(&h->h_loops, 2 * sizeof(int)));
  }
  catch(...)
  {
    mma_destroy(h);
    throw;
  }
  *out = h;
}

void mma_destroy(icarat_mma *h)
{
  if(!h)
    return;
  cudaSetDevice(h->device);
  if(h->stream)
    cudaStreamSynchronize(h->stream);
  for(double *p : {h->low, h->upp, h->alpha, h->beta, h->p0, h->q0, h->xold1,
                   h->xold2, h->pij, h->qij, h->stage, h->partials})
    dfree(p);
  dfree(h->loops);
  if(h->h_loops)
    cudaFreeHost(h->h_loops);
  if(h->stream && h->own_stream)
    cudaStreamDestroy(h->stream);
  delete h;
}

// Host-pointer update: stage, update on the device, copy x back.
int mma_update_host(icarat_mma *h, double *x, const double *dfdx, const double *gx,
                    const double *dgdx, const double *xmin, const double *xmax)
{
  const size_t n = h->n, m = h->m;
  double *dx = h->stage, *ddf = dx + n, *dmin = ddf + n, *dmax = dmin + n,
         *ddg = dmax + n;
  ICK(cudaMemcpyAsync(dx, x, sizeof(double) * n, cudaMemcpyHostToDevice, h->stream));
  ICK(cudaMemcpyAsync(ddf, dfdx, sizeof(double) * n, cudaMemcpyHostToDevice,
                      h->stream));
  ICK(cudaMemcpyAsync(dmin, xmin, sizeof(double) * n, cudaMemcpyHostToDevice,
                      h->stream));
  ICK(cudaMemcpyAsync(dmax, xmax, sizeof(double) * n, cudaMemcpyHostToDevice,
                      h->stream));
  ICK(cudaMemcpyAsync(ddg, dgdx, sizeof(double) * n * m, cudaMemcpyHostToDevice,
                      h->stream));
  int st = mma_update_device(h, dx, ddf, gx, ddg, dmin, dmax);
  ICK(cudaMemcpyAsync(x, dx, sizeof(double) * n, cudaMemcpyDeviceToHost, h->stream));
  ICK(cudaStreamSynchronize(h->stream));
  return st;
}

void mma_set_move(icarat_mma *h, double move) { h->move = move; }
int mma_last_newton(const icarat_mma *h) { return h->last_newton; }

// The state an MMA update carries to the next (asymptotes, the two previous
// designs, the iteration count that selects the asymptote rule), copied to
// (save) or from (load) host arrays of n entries.
void mma_state_io(icarat_mma *h, bool save, int *iter, double *low, double *upp,
                  double *xold1, double *xold2)
{
  const size_t bytes = sizeof(double) * h->n;
  double *dev[4] = {h->low, h->upp, h->xold1, h->xold2};
  double *host[4] = {low, upp, xold1, xold2};
  for(int q = 0; q < 4; q++)
    ICK(cudaMemcpyAsync(save ? host[q] : dev[q], save ? dev[q] : host[q], bytes,
                        save ? cudaMemcpyDeviceToHost : cudaMemcpyHostToDevice, h->stream));
  ICK(cudaStreamSynchronize(h->stream));
  if(save)
    *iter = h->iter;
  else
    h->iter = *iter;
}

} // namespace icarat_b200

using namespace icarat_b200;

extern "C" {

int icarat_mma_create(int device, int n, int m, double a, double c, double d,
                      icarat_mma **out)
{
  ICARAT_API_BEGIN
  IREQUIRE(out, ICARAT_ERR_ARG, "null output handle");
  mma_create(device, n, m, a, c, d, out, nullptr);
  return ICARAT_OK;
  ICARAT_API_END
}

int icarat_mma_destroy(icarat_mma *h)
{
  ICARAT_API_BEGIN
  mma_destroy(h);
  return ICARAT_OK;
  ICARAT_API_END
}

int icarat_mma_set_move_limit(icarat_mma *h, double move)
{
  ICARAT_API_BEGIN
  IREQUIRE(h, ICARAT_ERR_ARG, "null handle");
  h->move = move;
  return ICARAT_OK;
  ICARAT_API_END
}

int icarat_mma_set_asymptotes(icarat_mma *h, double init, double dec, double inc)
{
  ICARAT_API_BEGIN
  IREQUIRE(h, ICARAT_ERR_ARG, "null handle");
  h->asyminit = init;
  h->asymdec = dec;
  h->asyminc = inc;
  return ICARAT_OK;
  ICARAT_API_END
}

int icarat_mma_set_oscillation(icarat_mma *h, double albefa)
{
  ICARAT_API_BEGIN
  IREQUIRE(h, ICARAT_ERR_ARG, "null handle");
  h->albefa = albefa;
  return ICARAT_OK;
  ICARAT_API_END
}

int icarat_mma_update(icarat_mma *h, double *x, const double *dfdx, const double *gx,
                      const double *dgdx, const double *xmin, const double *xmax)
{
  ICARAT_API_BEGIN
  IREQUIRE(h && x && dfdx && gx && dgdx && xmin && xmax, ICARAT_ERR_ARG,
           "null argument");
  ICK(cudaSetDevice(h->device));
  return mma_update_host(h, x, dfdx, gx, dgdx, xmin, xmax);
  ICARAT_API_END
}

int icarat_mma_update_dev(icarat_mma *h, double *x, const double *dfdx,
                          const double *gx, const double *dgdx, const double *xmin,
                          const double *xmax)
{
  ICARAT_API_BEGIN
  IREQUIRE(h && x && dfdx && gx && dgdx && xmin && xmax, ICARAT_ERR_ARG,
           "null argument");
  ICK(cudaSetDevice(h->device));
  return mma_update_device(h, x, dfdx, gx, dgdx, xmin, xmax);
  ICARAT_API_END
}

int icarat_mma_last_loops(const icarat_mma *h, int *outer, int *newton)
{
  ICARAT_API_BEGIN
  IREQUIRE(h, ICARAT_ERR_ARG, "null handle");
  if(outer)
    *outer = h->last_outer;
  if(newton)
    *newton = h->last_newton;
  return ICARAT_OK;
  ICARAT_API_END
}

} // extern "C"
