// One design iteration with every array resident on the device: the loop body
// of sample/algorithm/opt-macro-oc/opt_macro_oc.cpp:83-172 (OC) and
// sample/algorithm/opt-macro-mma-nondesign/opt_macro_mma_nondesign.cpp:90-178
// (MMA), with the radius Filter or the Helmholtz PDE filter of
// opt_macro_oc.cpp:73-74 / opt_mma_Helmholtz.cpp:70-72 and an optional
// Heaviside threshold.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "internal.cuh"

namespace icarat_b200
{

int mma_update_device(icarat_mma *h, double *x, const double *dfdx, const double *gx,
                      const double *dgdx, const double *xmin, const double *xmax);
void mma_create(int device, int n, int m, double a, double c, double d,
                icarat_mma **out, cudaStream_t stream);
void mma_set_move(icarat_mma *h, double move);
int mma_last_newton(const icarat_mma *h);
void mma_state_io(icarat_mma *h, bool save, int *iter, double *low, double *upp,
                  double *xold1, double *xold2);

__global__ void k_fill(int n, double v, double *__restrict__ out)
{
  for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
      i += gridDim.x * blockDim.x)
    out[i] = v;
}

// v on kept elements, 0 on elements a selection removed (mask null: all kept)
__global__ void k_fill_kept(int n, double v, const uint8_t *__restrict__ emask,
                            double *__restrict__ out)
{
  for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
      i += gridDim.x * blockDim.x)
    out[i] = (emask && !emask[i]) ? 0.0 : v;
}

__global__ void k_sel_gather(int n, const int *__restrict__ map,
                             const double *__restrict__ in, double *__restrict__ out);
__global__ void k_sel_scatter(int n, const int *__restrict__ map,
                              const double *__restrict__ in, double *__restrict__ out);

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

void loop_free_domains(icarat_ctx *c);

int loop_init(icarat_ctx *c, const icarat_loop_opts *o, const double *x0)
{
  IREQUIRE(o->method == 0 || o->method == 1, ICARAT_ERR_ARG, "method must be 0 (OC) or 1 (MMA)");
  IREQUIRE(o->filter_kind == 0 || o->filter_kind == 1, ICARAT_ERR_ARG,
           "filter_kind must be 0 (radius) or 1 (Helmholtz)");
  IREQUIRE(!(c->sel && o->filter_kind == 1), ICARAT_ERR_UNSUPPORTED,
           "the Helmholtz filter is not available on a selected (sub-)mesh");
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
  L.object_f = 0.0;
  L.object_old = 0.0;
  loop_free_domains(c);
  if(o->filter_kind == 1)
    helm_setup(c, o->filter_radius);
  else
    filter_setup(c, o->filter_radius);
  elem_in(c, x0, true, L.x);
  if(c->sel && !L.d_sel)
    L.d_sel = dalloc(5 * (size_t)c->nelx_sel);
  note_launch();
  k_fill<<<eb(n), 256, 0, c->stream>>>(n, o->xmin, L.xmin);
  note_launch();
  k_fill<<<eb(n), 256, 0, c->stream>>>(n, o->xmax, L.xmax);
  ICK(cudaGetLastError());
  if(o->method == 1)
  {
    // MMASolver mma(nelx, 1) with SetMoveLimit (opt_mma_Helmholtz.cpp uses 0.2)
    // (on the kept elements of a selection: the reference's MMA has nelx of
    // the modified mesh variables)
    mma_create(c->device, abi_nelx(c), 1, 0.0, 100000.0, 0.0, &L.mma, c->stream);
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

__global__ void k_add(int n, const double *__restrict__ a, double *__restrict__ b)
{
  for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
      i += gridDim.x * blockDim.x)
    b[i] += a[i];
}

// dfds = dgds = 0 on non-design elements (opt_macro_mma_nondesign.cpp:161-166)
__global__ void k_zero_fixed(int n, const uint8_t *__restrict__ fixed, double *__restrict__ a,
                             double *__restrict__ b)
{
  for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
      i += gridDim.x * blockDim.x)
    if(fixed[i])
    {
      a[i] = 0.0;
      b[i] = 0.0;
    }
}

// volume of the thresholded design over the design IDs (all elements without
// domains) and the constraint of this step; sets V0 on the first step
static double loop_constraint(icarat_ctx *c)
{
  LoopState &L = c->loop;
  const int n = c->nelx;
  const double *w = L.d_volw;
  if(!w)
  {
    note_launch();
    k_fill_kept<<<eb(n), 256, 0, c->stream>>>(n, c->vol0, c->d_emask, L.tmp);
    w = L.tmp;
  }
  const double vol = device_dot(c, L.xthr, w, n);
  const bool mma = L.opts.method == 1;
  if(L.optstep == 1)
  {
    L.V0 = vol;
    return mma ? 0.0 : vol;
  }
  return mma ? vol / L.V0 - 1.0 : vol;
}

// threshold chain rule, transposed filter, non-design zeroing and the OC or
// MMA update; returns the update's status
static int loop_finish(icarat_ctx *c, double beta, double constraint, int *usteps)
{
  LoopState &L = c->loop;
  const int n = c->nelx;
  const icarat_loop_opts &o = L.opts;
  note_launch();
  k_mul2<<<eb(n), 256, 0, c->stream>>>(n, L.thrd, L.dfds, L.dgds);
  if(o.filter_kind == 1)
  {
    // densityFilter(dfds / dgds, .., true) (opt_mma_Helmholtz.cpp:150-151)
    int st1 = helm_filter(c, L.dfds, L.tmp, true, 0.0, 0, nullptr);
    int st2 = helm_filter(c, L.dgds, L.tmp2, true, 0.0, 0, nullptr);
    IREQUIRE(st1 >= 0 && st2 >= 0, st1 < 0 ? st1 : st2, "Helmholtz filter failed");
  }
  else
    // both transposed filters in one pass, into the spare buffers
    filter_trans2(c, L.dfds, L.dgds, L.tmp, L.tmp2);
  // the spare buffers become the sensitivities
  std::swap(L.dfds, L.tmp);
  std::swap(L.dgds, L.tmp2);
  if(L.d_fixed)
  {
    note_launch();
    k_zero_fixed<<<eb(n), 256, 0, c->stream>>>(n, L.d_fixed, L.dfds, L.dgds);
  }
  ICK(cudaGetLastError());
  int ust = ICARAT_OK;
  *usteps = 0;
  if(o.method == 1 && c->sel)
  {
    // MMA over the kept elements: gather, update, scatter the design back
    const int m = c->nelx_sel;
    double *sx = L.d_sel, *sdf = sx + m, *sdg = sx + 2L * m, *smin = sx + 3L * m,
           *smax = sx + 4L * m;
    const double *src[5] = {L.x, L.dfds, L.dgds, L.xmin, L.xmax};
    double *dst[5] = {sx, sdf, sdg, smin, smax};
    for(int q = 0; q < 5; q++)
    {
      note_launch();
      k_sel_gather<<<eb(m), 256, 0, c->stream>>>(m, c->d_sel_elem, src[q], dst[q]);
    }
    ICK(cudaGetLastError());
    double g = constraint;
    ust = mma_update_device(L.mma, sx, sdf, &g, sdg, smin, smax);
    *usteps = mma_last_newton(L.mma);
    note_launch();
    k_sel_scatter<<<eb(m), 256, 0, c->stream>>>(m, c->d_sel_elem, sx, L.x);
    ICK(cudaGetLastError());
  }
  else if(o.method == 1)
  {
    double g = constraint;
    ust = mma_update_device(L.mma, L.x, L.dfds, &g, L.dgds, L.xmin, L.xmax);
    *usteps = mma_last_newton(L.mma);
  }
  else
  {
    icarat_oc_opts oc{o.move, 0.5, 0.0, 1.0e4, 1.0e-5, 100, o.use_threshold, beta, o.T, 0};
    if(o.filter_kind == 1)
    {
      // after the swap L.tmp / L.tmp2 hold the unfiltered sensitivities, no
      // longer needed: they take the filtered and thresholded trials; the
      // element volumes go to c->d_e1
      note_launch();
      k_fill<<<eb(n), 256, 0, c->stream>>>(n, c->vol0, c->d_e1);
      ICK(cudaGetLastError());
      ust = oc_update_helm_dev(c, L.x, L.dfds, L.V0, L.dgds, L.xmin, L.xmax, &oc, usteps,
                               L.tmp, L.tmp2, c->d_e1);
    }
    else
      ust = oc_update_dev(c, L.x, L.dfds, L.V0, L.dgds, L.xmin, L.xmax, &oc, usteps);
  }
  ICK(cudaStreamSynchronize(c->stream));
  return ust;
}

static int step_status(int st, int ust)
{
  return st < 0 ? st : (ust < 0 ? ust : (st != ICARAT_OK ? st : ust));
}

// Rest of a design iteration after the solve (status st, info si):
// compliance, volume, sensitivities, transposed filter and the update.
int loop_post(icarat_ctx *c, int st, const icarat_solve_info &si, double beta,
              icarat_step_info *info)
{
  LoopState &L = c->loop;
  const icarat_loop_opts &o = L.opts;
  c->solved = true;
  c->have_u = true;
  c->last_info = si;
  const double compliance = compliance_dev(c);
  const double constraint = loop_constraint(c);
  sensitivity_dev(c, o.method == 1 ? 1.0 / L.V0 : 1.0, L.dfds, L.dgds);
  int usteps = 0;
  const int ust = loop_finish(c, beta, constraint, &usteps);
  L.object_f = compliance;
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
  return step_status(st, ust);
}

// A design iteration over several load cases (opt_multi_load.cpp:100-200):
// one solve per case on the same design (the multigrid hierarchy is built
// once), object_f = sum_lc u_lc . f_lc and dfds = sum_lc -(E'/E) u_lc Ke u_lc
// accumulated in case order, then the shared tail.  The constraint is the
// design-domain volume, as in that driver.
static int loop_step_cases(icarat_ctx *c, double beta, icarat_step_info *info)
{
  LoopState &L = c->loop;
  const int n = c->nelx;
  const double constraint = loop_constraint(c);
  double compliance = 0.0, relres = 0.0;
  int iterations = 0, st = ICARAT_OK;
  double *own = c->d_fext;
  try
  {
    for(int lc = 0; lc < L.ncases; lc++)
    {
      c->d_fext = L.d_cases + (size_t)lc * c->neq;
      build_rhs(c);
      // a warm start begins from this case's own last solution
      double *ucase = L.d_cases_u + (size_t)lc * c->neq;
      if(L.opts.solve.warm_start)
      {
        if(L.cases_have[lc])
          ICK(cudaMemcpyAsync(c->d_u, ucase, sizeof(double) * c->neq,
                              cudaMemcpyDeviceToDevice, c->stream));
        else
          ICK(cudaMemsetAsync(c->d_u, 0, sizeof(double) * c->neq, c->stream));
        c->have_u = L.cases_have[lc] != 0;
      }
      icarat_solve_info si{};
      const int s1 = solve_full(c, &L.opts.solve, c->d_rhs, c->d_u, &si);
      if(L.opts.solve.warm_start)
      {
        ICK(cudaMemcpyAsync(ucase, c->d_u, sizeof(double) * c->neq, cudaMemcpyDeviceToDevice,
                            c->stream));
        L.cases_have[lc] = 1;
      }
      if(s1 < 0 || (st >= 0 && s1 != ICARAT_OK))
        st = s1;
      c->solved = true;
      c->have_u = true;
      c->last_info = si;
      iterations += si.iterations;
      relres = relres > si.rel_residual ? relres : si.rel_residual;
      compliance += compliance_dev(c);
      // first case into dfds, later cases through the spare buffer
      sensitivity_dev(c, 1.0 / L.V0, lc == 0 ? L.dfds : L.tmp2, L.dgds);
      if(lc > 0)
      {
        note_launch();
        k_add<<<eb(n), 256, 0, c->stream>>>(n, L.tmp2, L.dfds);
        ICK(cudaGetLastError());
      }
    }
  }
  catch(...)
  {
    c->d_fext = own;
    throw;
  }
  c->d_fext = own;
  int usteps = 0;
  const int ust = loop_finish(c, beta, constraint, &usteps);
  L.object_f = compliance;
  if(info)
  {
    info->step = L.optstep;
    info->compliance = compliance;
    info->constraint = constraint;
    info->cg_iterations = iterations;
    info->cg_rel_residual = relres;
    info->update_steps = usteps;
    info->status = st != ICARAT_OK ? st : ust;
  }
  return step_status(st, ust);
}

int loop_step(icarat_ctx *c, icarat_step_info *info)
{
  const LoopState &L = c->loop;
  IREQUIRE(!L.init || L.opts.method == 1 || (L.ncases == 0 && !L.d_volw),
           ICARAT_ERR_UNSUPPORTED,
           "load cases and design domains take the MMA update (opt_multi_load.cpp, "
           "opt_macro_mma_nondesign.cpp)");
  const double beta = loop_pre(c);
  if(c->loop.ncases > 0)
    return loop_step_cases(c, beta, info);
  icarat_solve_info si{};
  const int st = solve_full(c, &c->loop.opts.solve, c->d_rhs, c->d_u, &si);
  return loop_post(c, st, si, beta, info);
}

// Load cases of a multi-load loop: ncases x numeq host vectors (the layout of
// icarat_fext), kept on the device in node layout; ncases = 0 returns to the
// context's own load.
int set_load_cases(icarat_ctx *c, int ncases, const double *fext)
{
  LoopState &L = c->loop;
  IREQUIRE(ncases >= 0 && (ncases == 0 || fext), ICARAT_ERR_ARG, "bad load cases");
  dfree(L.d_cases);
  dfree(L.d_cases_u);
  L.d_cases = L.d_cases_u = nullptr;
  L.cases_have.clear();
  L.ncases = 0;
  if(ncases == 0)
    return ICARAT_OK;
  L.d_cases = dalloc((size_t)ncases * c->neq);
  L.d_cases_u = dalloc((size_t)ncases * c->neq);
  L.cases_have.assign(ncases, 0);
  for(int lc = 0; lc < ncases; lc++)
    to_full(c, fext + (size_t)lc * c->numeq, L.d_cases + (size_t)lc * c->neq, true);
  ICK(cudaStreamSynchronize(c->stream));
  L.ncases = ncases;
  return ICARAT_OK;
}

// Design / non-design element IDs of the loop (the pair returned by
// getDesignNonDesignIDs, non_design_domain.hpp:9-53 and
// opt_macro_mma_nondesign.cpp:247-317): the volume constraint sums over the
// design IDs (NULL: every element), sensitivities are zeroed on the
// non-design IDs after the transposed filter.  Cleared by icarat_loop_init.
int loop_set_domains(icarat_ctx *c, const int *design_ids, int n_design,
                     const int *nondesign_ids, int n_nondesign)
{
  LoopState &L = c->loop;
  IREQUIRE(L.init, ICARAT_ERR_STATE, "icarat_loop_init first");
  IREQUIRE(n_design >= 0 && n_nondesign >= 0 && (n_design == 0 || design_ids) &&
               (n_nondesign == 0 || nondesign_ids),
           ICARAT_ERR_ARG, "bad domain lists");
  const int n = c->nelx, na = abi_nelx(c);
  // IDs are element numbers of the (selected) mesh; box ids inside
  auto box_id = [&](int id) { return c->sel ? c->sel_elem_h[id] : id; };
  std::vector<double> w(n, 0.0);
  if(!design_ids)
    for(int q = 0; q < na; q++)
      w[box_id(q)] = c->vol0;
  for(int q = 0; q < n_design; q++)
  {
    IREQUIRE(design_ids[q] >= 0 && design_ids[q] < na, ICARAT_ERR_ARG,
             "design ID out of range");
    w[box_id(design_ids[q])] = c->vol0;
  }
  std::vector<uint8_t> f(n, 0);
  for(int q = 0; q < n_nondesign; q++)
  {
    IREQUIRE(nondesign_ids[q] >= 0 && nondesign_ids[q] < na, ICARAT_ERR_ARG,
             "non-design ID out of range");
    f[box_id(nondesign_ids[q])] = 1;
  }
  if(!L.d_volw)
    L.d_volw = dalloc(n);
  if(!L.d_fixed)
    ICK(cudaMalloc(&L.d_fixed, n));
  ICK(cudaMemcpy(L.d_volw, w.data(), sizeof(double) * n, cudaMemcpyHostToDevice));
  ICK(cudaMemcpy(L.d_fixed, f.data(), n, cudaMemcpyHostToDevice));
  return ICARAT_OK;
}

void loop_free_domains(icarat_ctx *c)
{
  LoopState &L = c->loop;
  dfree(L.d_volw);
  dfree(L.d_fixed);
  L.d_volw = nullptr;
  L.d_fixed = nullptr;
}

// Optimize::isConvergence(epsilon, minstep) (src/optimization/opt_base.hpp:28-43)
// on the loop's objective: 0 when |object_old - object_f| / object_f < epsilon
// and optstep > minstep, else 1 with object_old = object_f.  The reference
// leaves object_old uninitialised before the first call; here it starts at 0,
// so the first call compares against |object_f| / object_f = 1.
int loop_is_convergence(icarat_ctx *c, double epsilon, double minstep, int *convergence)
{
  LoopState &L = c->loop;
  IREQUIRE(L.init, ICARAT_ERR_STATE, "icarat_loop_init first");
  IREQUIRE(L.optstep > 0, ICARAT_ERR_STATE, "icarat_loop_step first");
  if(std::fabs(L.object_old - L.object_f) / L.object_f < epsilon && L.optstep > minstep)
    *convergence = 0;
  else
  {
    L.object_old = L.object_f;
    *convergence = 1;
  }
  return ICARAT_OK;
}

// ---- loop snapshot (checkpoint / resume) ---------------------------------
// Binary file, native byte order: magic, layout version, grid and sizes, the
// loop options, the step counter, V0, the convergence test's objectives, the
// design x (box element layout), the MMA state (asymptotes, two previous
// designs, iteration count) and the displacement a warm start begins from.
// Load cases and design domains are the caller's configuration: set them
// again after icarat_loop_load, as after icarat_loop_init.
namespace
{
const char kSnapMagic[8] = {'I', 'C', 'R', 'L', 'O', 'O', 'P', '1'};
struct SnapHead
{
  char magic[8];
  int version, nx, ny, nz, nelx, neq, numeq, sel_nelx;
  int optstep, mma_iter, have_u, pad;
  double lx, ly, lz, V0, object_f, object_old;
  icarat_loop_opts opts;
};

struct File
{
  FILE *f;
  explicit File(FILE *p) : f(p) {}
  ~File()
  {
    if(f)
      fclose(f);
  }
};
} // namespace

int loop_save(icarat_ctx *c, const char *path)
{
  LoopState &L = c->loop;
  IREQUIRE(L.init, ICARAT_ERR_STATE, "icarat_loop_init first");
  SnapHead h{};
  std::memcpy(h.magic, kSnapMagic, 8);
  h.version = 2;
  h.nx = c->nx;
  h.ny = c->ny;
  h.nz = c->nz;
  h.nelx = c->nelx;
  h.neq = c->neq;
  h.numeq = c->numeq;
  h.sel_nelx = abi_nelx(c);
  h.optstep = L.optstep;
  h.mma_iter = -1;
  h.have_u = c->have_u ? 1 : 0;
  h.lx = c->lx;
  h.ly = c->ly;
  h.lz = c->lz;
  h.V0 = L.V0;
  h.object_f = L.object_f;
  h.object_old = L.object_old;
  h.opts = L.opts;
  const size_t n = c->nelx;
  std::vector<double> x(n), u(h.have_u ? (size_t)c->neq : 0);
  ICK(cudaMemcpyAsync(x.data(), L.x, sizeof(double) * n, cudaMemcpyDeviceToHost, c->stream));
  if(h.have_u)
    ICK(cudaMemcpyAsync(u.data(), c->d_u, sizeof(double) * c->neq, cudaMemcpyDeviceToHost,
                        c->stream));
  ICK(cudaStreamSynchronize(c->stream));
  std::vector<double> mma;
  if(L.mma)
  {
    const size_t m = abi_nelx(c);
    mma.resize(4 * m);
    mma_state_io(L.mma, true, &h.mma_iter, mma.data(), mma.data() + m, mma.data() + 2 * m,
                 mma.data() + 3 * m);
  }
  File f(std::fopen(path, "wb"));
  IREQUIRE(f.f != nullptr, ICARAT_ERR_ARG, std::string("cannot write ") + path);
  bool ok = std::fwrite(&h, sizeof(h), 1, f.f) == 1 &&
            std::fwrite(x.data(), sizeof(double), n, f.f) == n &&
            std::fwrite(mma.data(), sizeof(double), mma.size(), f.f) == mma.size() &&
            std::fwrite(u.data(), sizeof(double), u.size(), f.f) == u.size();
  IREQUIRE(ok, ICARAT_ERR_ARG, std::string("write failed: ") + path);
  return ICARAT_OK;
}

int loop_load(icarat_ctx *c, const char *path)
{
  File f(std::fopen(path, "rb"));
  IREQUIRE(f.f != nullptr, ICARAT_ERR_ARG, std::string("cannot read ") + path);
  SnapHead h{};
  IREQUIRE(std::fread(&h, sizeof(h), 1, f.f) == 1 && std::memcmp(h.magic, kSnapMagic, 8) == 0 &&
               h.version == 2,
           ICARAT_ERR_ARG, std::string("not a loop snapshot: ") + path);
  IREQUIRE(h.nx == c->nx && h.ny == c->ny && h.nz == c->nz && h.nelx == c->nelx &&
               h.neq == c->neq && h.numeq == c->numeq && h.sel_nelx == abi_nelx(c) &&
               h.lx == c->lx && h.ly == c->ly && h.lz == c->lz,
           ICARAT_ERR_ARG, "the snapshot belongs to another mesh or boundary conditions");
  const size_t n = c->nelx, m = abi_nelx(c);
  std::vector<double> x(n), mma(h.mma_iter >= 0 ? 4 * m : 0), u(h.have_u ? (size_t)h.neq : 0);
  bool ok = std::fread(x.data(), sizeof(double), n, f.f) == n &&
            std::fread(mma.data(), sizeof(double), mma.size(), f.f) == mma.size() &&
            std::fread(u.data(), sizeof(double), u.size(), f.f) == u.size();
  IREQUIRE(ok, ICARAT_ERR_ARG, std::string("truncated snapshot: ") + path);
  IREQUIRE((h.opts.method == 1) == (h.mma_iter >= 0), ICARAT_ERR_ARG, "inconsistent snapshot");
  // a fresh loop with the saved options, then the saved state on top; x0 of
  // loop_init is in the ABI's numbering, the saved x in box layout
  std::vector<double> x0(m);
  if(c->sel)
    for(size_t q = 0; q < m; q++)
      x0[q] = x[c->sel_elem_h[q]];
  else
    x0 = x;
  loop_init(c, &h.opts, x0.data());
  LoopState &L = c->loop;
  ICK(cudaMemcpyAsync(L.x, x.data(), sizeof(double) * n, cudaMemcpyHostToDevice, c->stream));
  if(h.have_u)
    ICK(cudaMemcpyAsync(c->d_u, u.data(), sizeof(double) * h.neq, cudaMemcpyHostToDevice,
                        c->stream));
  ICK(cudaStreamSynchronize(c->stream));
  c->have_u = h.have_u != 0;
  L.optstep = h.optstep;
  L.V0 = h.V0;
  L.object_f = h.object_f;
  L.object_old = h.object_old;
  if(L.mma)
    mma_state_io(L.mma, false, &h.mma_iter, mma.data(), mma.data() + m, mma.data() + 2 * m,
                 mma.data() + 3 * m);
  return ICARAT_OK;
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
  elem_out(c, src, out, true);
  return ICARAT_OK;
}

} // namespace icarat_b200
