// Optimality-criteria update (OC::UpdateVariables,
// src/optimization/opt-solver/OCSolver.hpp:21-68) with the volume functor of
// the sample drivers, g(x) = sum_i thr(filter(x))_i v_i
// (sample/algorithm/opt-macro-oc/opt_macro_oc.cpp:153-164).
//
// The whole bisection runs in one cooperative launch: per step every block
// writes its trial densities, the grid synchronises, every block filters its
// elements and writes one partial volume, the grid synchronises, and every
// block sums all partials in the same fixed order, so every block takes the
// same lambda decision without another barrier or a host round trip.
#include <cooperative_groups.h>

#include <cmath>

#include "internal.cuh"

namespace cg = cooperative_groups;

namespace icarat_b200
{

struct OcArgs
{
  int nx, ny, nz, nelx;
  int nofs;
  const int *ofs;
  const double *w;
  const double *x, *dfdx, *dgdx, *xmin, *xmax;
  double *xk;        // trial densities (nelx)
  double *partials;  // gridDim.x
  double *result;    // [0] steps, [1] lambda
  double move, iota, lmin, lmax, leps, g, vol, beta, T;
  int maxiter, use_thr;
  const uint8_t *emask; // elements kept by a selection (null: all)
};

__device__ __forceinline__ double oc_trial(const OcArgs &a, int i, double lambda)
{
  const double x = a.x[i];
  const double v = -a.dfdx[i] / (a.dgdx[i] * lambda);
  const double vp = v > 0.0 ? v : 0.0;
  // pow(v, 0.5) of the reference is the correctly rounded square root
  double xn = (a.iota == 0.5 ? sqrt(vp) : pow(vp, a.iota)) * x;
  const double lo0 = (1.0 - a.move) * x, hi0 = (1.0 + a.move) * x;
  const double lo = a.xmin[i] > lo0 ? a.xmin[i] : lo0;
  const double hi = a.xmax[i] < hi0 ? a.xmax[i] : hi0;
  if(xn < lo)
    xn = lo;
  else if(xn > hi)
    xn = hi;
  return xn;
}

__global__ void __launch_bounds__(256) k_oc_bisect(OcArgs a)
{
  cg::grid_group grid = cg::this_grid();
  __shared__ double sh[32];
  __shared__ double s_total;
  double l0 = a.lmin, l1 = a.lmax;
  int counter = 0;
  const double tb = a.use_thr ? tanh(a.T * a.beta) : 1.0;
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  const int stride = gridDim.x * blockDim.x;
  double lambda = 0.0;
  while((l1 - l0) / (l1 + l0) > a.leps && a.maxiter > counter)
  {
    lambda = 0.5 * (l1 + l0);
    for(int e = tid; e < a.nelx; e += stride)
      a.xk[e] = (a.emask && !a.emask[e]) ? 0.0 : oc_trial(a, e, lambda);
    grid.sync();
    double part = 0.0;
    for(int e = tid; e < a.nelx; e += stride)
    {
      if(a.emask && !a.emask[e])
        continue;
      const int i = e % a.nx, j = (e / a.nx) % a.ny, k = e / (a.nx * a.ny);
      double aa = 0.0, bb = 0.0;
      for(int q = 0; q < a.nofs; q++)
      {
        const int ii = i + a.ofs[3 * q], jj = j + a.ofs[3 * q + 1],
                  kk = k + a.ofs[3 * q + 2];
        if(ii < 0 || ii >= a.nx || jj < 0 || jj >= a.ny || kk < 0 || kk >= a.nz)
          continue;
        const long f = ii + (long)jj * a.nx + (long)kk * a.nx * a.ny;
        if(a.emask && !a.emask[f])
          continue;
        const double wq = a.w[q];
        aa = __dadd_rn(aa, wq);
        // written by other blocks in this launch: bypass L1
        bb = __dadd_rn(bb, __dmul_rn(wq, __ldcg(a.xk + f)));
      }
      double rho = __ddiv_rn(bb, aa);
      if(a.use_thr)
        rho = 0.5 * (tb + tanh(a.beta * (rho - a.T))) / tb;
      part += rho * a.vol;
    }
    double v[1] = {part};
    block_sum<1>(v, sh);
    if(threadIdx.x == 0)
      a.partials[blockIdx.x] = v[0];
    grid.sync();
    double t[1];
    sum_partials<1>(a.partials, gridDim.x, t, sh);
    if(threadIdx.x == 0)
      s_total = t[0];
    __syncthreads();
    if(s_total - a.g > 0.0)
      l0 = lambda;
    else
      l1 = lambda;
    counter++;
  }
  if(blockIdx.x == 0 && threadIdx.x == 0)
  {
    a.result[0] = counter;
    a.result[1] = lambda;
  }
}

// one trial design of the bisection (the Helmholtz volume functor's input)
__global__ void k_oc_trial(OcArgs a, double lambda)
{
  for(int e = blockIdx.x * blockDim.x + threadIdx.x; e < a.nelx;
      e += gridDim.x * blockDim.x)
    a.xk[e] = (a.emask && !a.emask[e]) ? 0.0 : oc_trial(a, e, lambda);
}

__global__ void k_oc_fill(int n, double v, double *__restrict__ out)
{
  for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    out[i] = v;
}

// x <- last trial (zeros when no step ran, like the reference's xkp1)
__global__ void k_oc_finish(int n, const double *__restrict__ xk, int steps,
                            double *__restrict__ x)
{
  for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
      i += gridDim.x * blockDim.x)
    x[i] = steps > 0 ? xk[i] : 0.0;
}

int oc_update_dev(icarat_ctx *c, double *x, const double *dfdx, double g,
                  const double *dgdx, const double *xmin, const double *xmax,
                  const icarat_oc_opts *o, int *steps)
{
  IREQUIRE(o->filter_kind == 0 || o->filter_kind == 1, ICARAT_ERR_ARG,
           "filter_kind must be 0 (radius) or 1 (Helmholtz)");
  if(o->filter_kind == 1)
  {
    // the Helmholtz functor of opt_macro_oc.cpp:153-164 on the set-up's
    // work vectors: filtered trial, thresholded trial, element volumes
    HelmState &H = c->helm;
    IREQUIRE(H.d_oc != nullptr, ICARAT_ERR_STATE,
             "the OC volume functor needs icarat_helmholtz_setup");
    const int n = c->nelx;
    note_launch();
    k_oc_fill<<<(n + 255) / 256, 256, 0, c->stream>>>(n, c->vol0, H.d_oc + 2L * n);
    ICK(cudaGetLastError());
    return oc_update_helm_dev(c, x, dfdx, g, dgdx, xmin, xmax, o, steps, H.d_oc, H.d_oc + n,
                              H.d_oc + 2L * n);
  }
  IREQUIRE(c->filt.d_w != nullptr, ICARAT_ERR_STATE,
           "the OC volume functor needs icarat_filter_setup");
  IREQUIRE(c->filt.radius >= 1.0e-10, ICARAT_ERR_FILTER,
           "coefficient aa is too small in the density filter");
  IREQUIRE(o->maxiter >= 0 && o->lambda_max + o->lambda_min > 0, ICARAT_ERR_ARG,
           "bad OC parameters");
  OcArgs a;
  a.nx = c->nx;
  a.ny = c->ny;
  a.nz = c->nz;
  a.nelx = c->nelx;
  a.nofs = c->filt.nofs;
  a.ofs = c->filt.d_ofs;
  a.w = c->filt.d_w;
  a.x = x;
  a.dfdx = dfdx;
  a.dgdx = dgdx;
  a.xmin = xmin;
  a.xmax = xmax;
  a.xk = c->d_e2;
  a.partials = c->d_partials;
  a.result = c->d_scalar;
  a.move = o->move;
  a.iota = o->iota;
  a.lmin = o->lambda_min;
  a.lmax = o->lambda_max;
  a.leps = o->lambda_eps;
  a.g = g;
  a.vol = c->vol0;
  a.beta = o->beta;
  a.T = o->T;
  a.maxiter = o->maxiter;
  a.use_thr = o->use_threshold ? 1 : 0;
  a.emask = c->d_emask;
  int per_sm = 0, sms = 0;
  ICK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_oc_bisect, 256, 0));
  ICK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device));
  int blocks = sms * (per_sm > 2 ? 2 : per_sm);
  const int need = (c->nelx + 255) / 256;
  if(blocks > need)
    blocks = need;
  if(blocks > kMaxRedBlocks)
    blocks = kMaxRedBlocks;
  IREQUIRE(blocks >= 1, ICARAT_ERR_CUDA, "no co-resident blocks for the OC kernel");
  void *args[] = {&a};
  note_launch();
  ICK(cudaLaunchCooperativeKernel((void *)k_oc_bisect, dim3(blocks), dim3(256), args,
                                  0, c->stream));
  ICK(cudaMemcpyAsync(c->h_scalar, c->d_scalar, 2 * sizeof(double),
                      cudaMemcpyDeviceToHost, c->stream));
  ICK(cudaStreamSynchronize(c->stream));
  const int nsteps = (int)c->h_scalar[0];
  note_launch();
  k_oc_finish<<<(c->nelx + 255) / 256, 256, 0, c->stream>>>(c->nelx, c->d_e2, nsteps,
                                                            x);
  ICK(cudaGetLastError());
  if(steps)
    *steps = nsteps;
  return nsteps >= o->maxiter ? ICARAT_WARN_MAXITER : ICARAT_OK;
}

// The same bisection with the volume functor of opt_macro_oc.cpp:153-164 on
// the Helmholtz filter: g(x) = sum_i thr(H(x))_i v_i needs a nodal solve
// per step, so the host drives the steps (trial kernel, Helmholtz filter,
// threshold, volume dot) and takes each lambda decision.  fil and thr are
// nelx work vectors, vol the element volumes (nelx).
int oc_update_helm_dev(icarat_ctx *c, double *x, const double *dfdx, double g,
                       const double *dgdx, const double *xmin, const double *xmax,
                       const icarat_oc_opts *o, int *steps, double *fil, double *thr,
                       const double *vol)
{
  IREQUIRE(c->helm.d_coef != nullptr, ICARAT_ERR_STATE,
           "the Helmholtz OC volume functor needs the Helmholtz filter set up");
  IREQUIRE(o->maxiter >= 0 && o->lambda_max + o->lambda_min > 0, ICARAT_ERR_ARG,
           "bad OC parameters");
  OcArgs a{};
  a.nelx = c->nelx;
  a.x = x;
  a.dfdx = dfdx;
  a.dgdx = dgdx;
  a.xmin = xmin;
  a.xmax = xmax;
  a.xk = c->d_e2;
  a.move = o->move;
  a.iota = o->iota;
  a.emask = c->d_emask;
  const int n = c->nelx;
  const int blocks = (n + 255) / 256 > 4 * c->sm_count ? 4 * c->sm_count : (n + 255) / 256;
  double l0 = o->lambda_min, l1 = o->lambda_max;
  int counter = 0;
  while((l1 - l0) / (l1 + l0) > o->lambda_eps && o->maxiter > counter)
  {
    const double lambda = 0.5 * (l1 + l0);
    note_launch();
    k_oc_trial<<<blocks, 256, 0, c->stream>>>(a, lambda);
    ICK(cudaGetLastError());
    const int st = helm_filter(c, a.xk, fil, false, 0.0, 0, nullptr);
    if(st < 0)
      return st;
    const double *t = fil;
    if(o->use_threshold)
    {
      threshold_dev(c, fil, o->beta, o->T, thr, false);
      t = thr;
    }
    if(device_dot(c, t, vol, n) - g > 0.0)
      l0 = lambda;
    else
      l1 = lambda;
    counter++;
  }
  note_launch();
  k_oc_finish<<<blocks, 256, 0, c->stream>>>(n, c->d_e2, counter, x);
  ICK(cudaGetLastError());
  ICK(cudaStreamSynchronize(c->stream));
  if(steps)
    *steps = counter;
  return counter >= o->maxiter ? ICARAT_WARN_MAXITER : ICARAT_OK;
}

} // namespace icarat_b200
