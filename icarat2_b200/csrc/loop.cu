// One design iteration with every array resident on the device: the loop body
// of sample/algorithm/opt-macro-oc/opt_macro_oc.cpp:83-172 (OC) and
// sample/algorithm/opt-macro-mma-nondesign/opt_macro_mma_nondesign.cpp:90-178
// (MMA), with the radius Filter or the Helmholtz PDE filter of
// opt_macro_oc.cpp:73-74 / opt_mma_Helmholtz.cpp:70-72 and an optional
// Heaviside threshold.
#include <cmath>

#include "internal.cuh"

namespace icarat_b200
{

int mma_update_device(icarat_mma *h, double *x, const double *dfdx, const double *gx,
                      const double *dgdx, const double *xmin, const double *xmax);
void mma_create(int device, int n, int m, double a, double c, double d,
                icarat_mma **out, cudaStream_t stream);
void mma_set_move(icarat_mma *h, double move);
int mma_last_newton(const icarat_mma *h);

__global__ void k_fill(int n, double v, double *__restrict__ out)
{
  for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
      i += gridDim.x * blockDim.x)
    out[i] = v;
}

__global__ void k_mul2(int n, const double *__restrict__ s, double *__restrict__ a,
                       double *__restrict__ b)
{
  for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
      i += gridDim.x * blockDim.x)
  {
    a[i] *= s[i];
    b[i] *= s[i];
  }
}

__global__ void k_sub(int n, const double *__restrict__ a, const double *__restrict__ b,
                      double *__restrict__ out)
{
  for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
      i += gridDim.x * blockDim.x)
    out[i] = a[i] - b[i];
}

// rhs = fext - fint (LinearAnalysis::solve, src/analysis/linear.hpp:73-80)
void build_rhs(icarat_ctx *c)
{
  if(c->has_uD)
  {
    launch_fint(c, c->d_v1);
    note_launch();
    k_sub<<<(c->neq + 255) / 256, 256, 0, c->stream>>>(c->neq, c->d_fext, c->d_v1,
                                                       c->d_rhs);
  }
  else
    ICK(cudaMemcpyAsync(c->d_rhs, c->d_fext, sizeof(double) * c->neq,
                        cudaMemcpyDeviceToDevice, c->stream));
  ICK(cudaGetLastError());
}

static int eb(int n) { return (n + 255) / 256 > 0 ? (n + 255) / 256 : 1; }

int loop_init(icarat_ctx *c, const icarat_loop_opts *o, const double *x0)
{
  IREQUIRE(o->method == 0 || o->method == 1, ICARAT_ERR_ARG, "method must be 0 (OC) or 1 (MMA)");
  IREQUIRE(o->filter_kind == 0 || o->filter_kind == 1, ICARAT_ERR_ARG,
           "filter_kind must be 0 (radius) or 1 (Helmholtz)");
  LoopState &L = c->loop;
  const int n = c->nelx;
  if(!L.x)
  {
    for(double **p : {&L.x, &L.xfil, &L.xthr, &L.thrd, &L.dfds, &L.dgds, &L.tmp, &L.tmp2,
                      &L.xmin, &L.xmax})
      *p = dalloc(n);
  }
  if(L.mma)
  {
    icarat_mma_destroy(L.mma);
    L.mma = nullptr;
  }
  L.opts = *o;
  L.optstep = 0;
  L.V0 = 0.0;
  if(o->filter_kind == 1)
    helm_setup(c, o->filter_radius);
  else
    filter_setup(c, o->filter_radius);
  ICK(cudaMemcpyAsync(L.x, x0, sizeof(double) * n, cudaMemcpyHostToDevice, c->stream));
  note_launch();
  k_fill<<<eb(n), 256, 0, c->stream>>>(n, o->xmin, L.xmin);
  note_launch();
  k_fill<<<eb(n), 256, 0, c->stream>>>(n, o->xmax, L.xmax);
  ICK(cudaGetLastError());
  if(o->method == 1)
  {
    // MMASolver mma(nelx, 1) with SetMoveLimit (opt_mma_Helmholtz.cpp uses 0.2)
    mma_create(c->device, n, 1, 0.0, 100000.0, 0.0, &L.mma, c->stream);
    mma_set_move(L.mma, o->move);
  }
  ICK(cudaStreamSynchronize(c->stream));
  L.init = true;
  return ICARAT_OK;
}

// First part of a design iteration: filter -> threshold -> element design ->
// right-hand side.  Returns the threshold sharpness beta of this step.
double loop_pre(icarat_ctx *c)
{
  LoopState &L = c->loop;
  IREQUIRE(L.init, ICARAT_ERR_STATE, "icarat_loop_init first");
  const int n = c->nelx;
  const icarat_loop_opts &o = L.opts;
  L.optstep++;
  // filter -> threshold -> element design
  if(o.filter_kind == 1)
  {
    const int st = helm_filter(c, L.x, L.xfil, false, 0.0, 0, nullptr);
    IREQUIRE(st >= 0, st, "Helmholtz filter failed");
  }
  else
    filter_apply(c, L.x, L.xfil, false);
  double beta = std::pow(2.0, (int)(L.optstep / 40));
  beta = beta < 16.0 ? beta : 16.0;
  if(o.use_threshold)
  {
    threshold_dev(c, L.xfil, beta, o.T, L.xthr, false);
    threshold_dev(c, L.xfil, beta, o.T, L.thrd, true);
  }
  else
  {
    ICK(cudaMemcpyAsync(L.xthr, L.xfil, sizeof(double) * n, cudaMemcpyDeviceToDevice,
                        c->stream));
    note_launch();
    k_fill<<<eb(n), 256, 0, c->stream>>>(n, 1.0, L.thrd);
  }
  set_design_device(c, L.xthr);
  build_rhs(c);
  return beta;
}

// Rest of a design iteration after the solve (status st, info si):
// compliance, volume, sensitivities, transposed filter and the update.
int loop_post(icarat_ctx *c, int st, const icarat_solve_info &si, double beta,
              icarat_step_info *info)
{
  LoopState &L = c->loop;
  const int n = c->nelx;
  const icarat_loop_opts &o = L.opts;
  c->solved = true;
  c->last_info = si;
  // objective and constraint
  const double compliance = compliance_dev(c);
  note_launch();
  k_fill<<<eb(n), 256, 0, c->stream>>>(n, c->vol0, L.tmp);
  const double vol = device_dot(c, L.xthr, L.tmp, n);
  double constraint;
  if(L.optstep == 1)
  {
    L.V0 = vol;
    constraint = (o.method == 1) ? 0.0 : vol;
  }
  else
    constraint = (o.method == 1) ? vol / L.V0 - 1.0 : vol;
  // sensitivities, threshold chain rule, transposed filter
  sensitivity_dev(c, o.method == 1 ? 1.0 / L.V0 : 1.0, L.dfds, L.dgds);
  note_launch();
  k_mul2<<<eb(n), 256, 0, c->stream>>>(n, L.thrd, L.dfds, L.dgds);
  // both transposed filters in one pass, into the spare buffers, which then
  // become the sensitivities
  if(o.filter_kind == 1)
  {
    // densityFilter(dfds / dgds, .., true) (opt_mma_Helmholtz.cpp:150-151)
    int st1 = helm_filter(c, L.dfds, L.tmp, true, 0.0, 0, nullptr);
    int st2 = helm_filter(c, L.dgds, L.tmp2, true, 0.0, 0, nullptr);
    IREQUIRE(st1 >= 0 && st2 >= 0, st1 < 0 ? st1 : st2, "Helmholtz filter failed");
  }
  else
    filter_trans2(c, L.dfds, L.dgds, L.tmp, L.tmp2);
  std::swap(L.dfds, L.tmp);
  std::swap(L.dgds, L.tmp2);
  // update
  int ust = ICARAT_OK, usteps = 0;
  if(o.method == 1)
  {
    double g = constraint;
    ust = mma_update_device(L.mma, L.x, L.dfds, &g, L.dgds, L.xmin, L.xmax);
    usteps = mma_last_newton(L.mma);
  }
  else
  {
    icarat_oc_opts oc{o.move, 0.5, 0.0, 1.0e4, 1.0e-5, 100, o.use_threshold, beta, o.T};
    if(o.filter_kind == 1)
    {
      // after the swap L.tmp / L.tmp2 hold the unfiltered sensitivities, no
      // longer needed: they take the filtered and thresholded trials; the
      // element volumes go to c->d_e1
      note_launch();
      k_fill<<<eb(n), 256, 0, c->stream>>>(n, c->vol0, c->d_e1);
      ICK(cudaGetLastError());
      ust = oc_update_helm_dev(c, L.x, L.dfds, L.V0, L.dgds, L.xmin, L.xmax, &oc, &usteps,
                               L.tmp, L.tmp2, c->d_e1);
    }
    else
      ust = oc_update_dev(c, L.x, L.dfds, L.V0, L.dgds, L.xmin, L.xmax, &oc, &usteps);
  }
  ICK(cudaStreamSynchronize(c->stream));
  if(info)
  {
    info->step = L.optstep;
    info->compliance = compliance;
    info->constraint = constraint;
    info->cg_iterations = si.iterations;
    info->cg_rel_residual = si.rel_residual;
    info->update_steps = usteps;
    info->status = st != ICARAT_OK ? st : ust;
  }
  return st < 0 ? st : (ust < 0 ? ust : (st != ICARAT_OK ? st : ust));
}

int loop_step(icarat_ctx *c, icarat_step_info *info)
{
  const double beta = loop_pre(c);
  icarat_solve_info si{};
  const int st = solve_full(c, &c->loop.opts.solve, c->d_rhs, c->d_u, &si);
  return loop_post(c, st, si, beta, info);
}

int loop_get(icarat_ctx *c, int which, double *out)
{
  LoopState &L = c->loop;
  IREQUIRE(L.init, ICARAT_ERR_STATE, "icarat_loop_init first");
  const double *src = nullptr;
  switch(which)
  {
  case 0: src = L.x; break;
  case 1: src = L.xfil; break;
  case 2: src = L.xthr; break;
  case 3: src = L.dfds; break;
  case 4: src = L.dgds; break;
  default: throw Error{ICARAT_ERR_ARG, "which must be 0..4"};
  }
  ICK(cudaMemcpyAsync(out, src, sizeof(double) * c->nelx, cudaMemcpyDeviceToHost,
                      c->stream));
  ICK(cudaStreamSynchronize(c->stream));
  return ICARAT_OK;
}

} // namespace icarat_b200
