// extern "C" entry points of include/icarat_gpu.h.  Each one converts C++
// errors into a status code; host pointers are staged through device buffers
// of the context.
#include <vector>
#include <atomic>
#include <cstring>
#include <string>

#include "internal.cuh"

int icarat_ctx_create_impl(const icarat_grid *grid, const icarat_material *mat,
                           const icarat_bc *bc, int device, icarat_ctx **out);
int icarat_ctx_create_sel_impl(const icarat_grid *grid, const icarat_material *mat,
                               const icarat_bc *bc, int nsel, const double *boxes,
                               int device, icarat_ctx **out);
int icarat_ctx_destroy_impl(icarat_ctx *c);

namespace icarat_b200
{
static thread_local std::string g_last_error;
void set_last_error(const std::string &msg) { g_last_error = msg; }

static std::atomic<unsigned long long> g_launches{0};
static thread_local bool g_capturing = false;
void note_launch(unsigned long long n)
{
  if(!g_capturing)
    g_launches += n;
}
void set_capturing(bool on) { g_capturing = on; }

void build_rhs(icarat_ctx *c);
int loop_init(icarat_ctx *c, const icarat_loop_opts *o, const double *x0);
int loop_is_convergence(icarat_ctx *c, double epsilon, double minstep, int *convergence);
int loop_save(icarat_ctx *c, const char *path);
int loop_load(icarat_ctx *c, const char *path);
int loop_step(icarat_ctx *c, icarat_step_info *info);
int loop_get(icarat_ctx *c, int which, double *out);
int set_load_cases(icarat_ctx *c, int ncases, const double *fext);
int loop_set_domains(icarat_ctx *c, const int *design_ids, int n_design,
                     const int *nondesign_ids, int n_nondesign);
void sensitivity_filter_dev(icarat_ctx *c, const double *s, const double *df,
                            double *out);

static double *stage(icarat_ctx *c, int k)
{
  if(!c->d_stage)
    c->d_stage = dalloc(6 * (size_t)c->nelx);
  return c->d_stage + (size_t)k * c->nelx;
}

static void h2d(icarat_ctx *c, double *dst, const double *src, size_t n)
{
  ICK(cudaMemcpyAsync(dst, src, sizeof(double) * n, cudaMemcpyHostToDevice, c->stream));
}

static void d2h(icarat_ctx *c, double *dst, const double *src, size_t n)
{
  ICK(cudaMemcpyAsync(dst, src, sizeof(double) * n, cudaMemcpyDeviceToHost, c->stream));
  ICK(cudaStreamSynchronize(c->stream));
}

static void check_ctx(const icarat_ctx *c)
{
  IREQUIRE(c != nullptr, ICARAT_ERR_ARG, "null context");
  ICK(cudaSetDevice(c->device));
}

static void no_selection(const icarat_ctx *c, const char *what)
{
  IREQUIRE(!c->sel, ICARAT_ERR_UNSUPPORTED,
           std::string(what) + " is not available on a selected (sub-)mesh");
}

static const icarat_solve_opts kDefaultSolve = {ICARAT_SOLVER_JACOBI_PCG, 1.0e-10,
                                                10000, 4, 2, 0};

} // namespace icarat_b200

using namespace icarat_b200;

// Average CUDA-event time of `launch` on the context's stream over reps
// launches, each preceded (outside its events) by a write of 256 MiB that
// evicts the L2, so every launch reads its operands from HBM.
template <typename F> static double time_cold(icarat_ctx *c, int reps, F &&launch)
{
  const size_t flush_bytes = 256ul << 20;
  void *flush = nullptr;
  ICK(cudaMalloc(&flush, flush_bytes));
  std::vector<cudaEvent_t> ev(2 * (size_t)reps);
  for(auto &e : ev)
    ICK(cudaEventCreate(&e));
  for(int r = 0; r < reps; r++)
  {
    ICK(cudaMemsetAsync(flush, r & 0xff, flush_bytes, c->stream));
    ICK(cudaEventRecord(ev[2 * r], c->stream));
    launch();
    ICK(cudaEventRecord(ev[2 * r + 1], c->stream));
  }
  ICK(cudaStreamSynchronize(c->stream));
  double total = 0.0;
  for(int r = 0; r < reps; r++)
  {
    float ms = 0.f;
    ICK(cudaEventElapsedTime(&ms, ev[2 * r], ev[2 * r + 1]));
    total += ms;
  }
  for(auto &e : ev)
    cudaEventDestroy(e);
  cudaFree(flush);
  return total / reps;
}

extern "C" {

// ICARAT_ABI_VERSION of the header the library was built with
int icarat_version(void) { return ICARAT_ABI_VERSION; }

int icarat_kernel_launches(unsigned long long *count)
{
  ICARAT_API_BEGIN
  IREQUIRE(count, ICARAT_ERR_ARG, "null argument");
  *count = g_launches.load();
  return ICARAT_OK;
  ICARAT_API_END
}

int icarat_mg_coarse_check(icarat_ctx *c, int mg_levels, double *rel_residual,
                           int *n_coarse)
{
  ICARAT_API_BEGIN
  check_ctx(c);
  IREQUIRE(rel_residual, ICARAT_ERR_ARG, "bad argument");
  IREQUIRE(c->design_set, ICARAT_ERR_STATE, "set the design first");
  *rel_residual = mg_coarse_check(c, mg_levels, n_coarse);
  return ICARAT_OK;
  ICARAT_API_END
}

int icarat_mg_level_apply(icarat_ctx *c, const icarat_solve_opts *opts, int level,
                          const double *x, double *y)
{
  ICARAT_API_BEGIN
  check_ctx(c);
  IREQUIRE(opts && x && y, ICARAT_ERR_ARG, "bad argument");
  IREQUIRE(c->design_set, ICARAT_ERR_STATE, "set the design first");
  mg_level_apply(c, opts, level, x, y);
  return ICARAT_OK;
  ICARAT_API_END
}

int icarat_time_operator(icarat_ctx *c, int reps, double *ms_per_launch)
{
  ICARAT_API_BEGIN
  check_ctx(c);
  IREQUIRE(reps > 0 && ms_per_launch, ICARAT_ERR_ARG, "bad argument");
  IREQUIRE(c->design_set, ICARAT_ERR_STATE, "set the design first");
  GridDev g{c->nx, c->ny, c->nz, c->NX, c->NY, c->NZ, c->numnp, c->nelx};
  // warm-up launch, then reps launches of the FP64 stencil y = K u, each
  // after a write of 256 MiB that evicts the 126 MB L2 (cold caches)
  launch_apply_K(c, g, c->d_E, c->d_fix, c->d_u, c->d_Ap, nullptr);
  *ms_per_launch = time_cold(c, reps, [&] {
    launch_apply_K(c, g, c->d_E, c->d_fix, c->d_u, c->d_Ap, nullptr);
  });
  return ICARAT_OK;
  ICARAT_API_END
}

const char *icarat_last_error(void) { return g_last_error.c_str(); }

const char *icarat_status_string(int s)
{
  switch(s)
  {
  case ICARAT_OK: return "ok";
  case ICARAT_WARN_MAXITER: return "iteration cap reached";
  case ICARAT_WARN_STAGNATION: return "residual stagnated";
  case ICARAT_ERR_ARG: return "bad argument";
  case ICARAT_ERR_CUDA: return "CUDA error";
  case ICARAT_ERR_NAN: return "non-finite value";
  case ICARAT_ERR_STATE: return "call order violated";
  case ICARAT_ERR_FILTER: return "filter weight sum too small";
  case ICARAT_ERR_UNSUPPORTED: return "unsupported";
  case ICARAT_ERR_NOMEM: return "out of memory";
  default: return "unknown status";
  }
}

int icarat_ctx_create(const icarat_grid *grid, const icarat_material *mat,
                      const icarat_bc *bc, int device, icarat_ctx **out)
{
  ICARAT_API_BEGIN
  return icarat_ctx_create_impl(grid, mat, bc, device, out);
  ICARAT_API_END
}

int icarat_ctx_create_selection(const icarat_grid *grid, const icarat_material *mat,
                                const icarat_bc *bc, int nsel, const double *boxes,
                                int device, icarat_ctx **out)
{
  ICARAT_API_BEGIN
  IREQUIRE(nsel >= 1 && boxes, ICARAT_ERR_ARG, "a selection needs at least one box");
  return icarat_ctx_create_sel_impl(grid, mat, bc, nsel, boxes, device, out);
  ICARAT_API_END
}

int icarat_selection_ids(const icarat_ctx *c, int *node_ids, int *elem_ids)
{
  ICARAT_API_BEGIN
  IREQUIRE(c, ICARAT_ERR_ARG, "null context");
  if(c->sel)
  {
    if(node_ids)
      std::memcpy(node_ids, c->sel_node_h.data(), sizeof(int) * c->sel_node_h.size());
    if(elem_ids)
      std::memcpy(elem_ids, c->sel_elem_h.data(), sizeof(int) * c->sel_elem_h.size());
  }
  else
  {
    for(int n = 0; node_ids && n < c->numnp; n++)
      node_ids[n] = n;
    for(int e = 0; elem_ids && e < c->nelx; e++)
      elem_ids[e] = e;
  }
  return ICARAT_OK;
  ICARAT_API_END
}

int icarat_ctx_destroy(icarat_ctx *c)
{
  ICARAT_API_BEGIN
  release_graphs(c);
  return icarat_ctx_destroy_impl(c);
  ICARAT_API_END
}

int icarat_sizes(const icarat_ctx *c, int *numnp, int *nelx, int *neq, int *numeq)
{
  ICARAT_API_BEGIN
  IREQUIRE(c, ICARAT_ERR_ARG, "null context");
  if(numnp)
    *numnp = c->sel ? c->numnp_sel : c->numnp;
  if(nelx)
    *nelx = abi_nelx(c);
  if(neq)
    *neq = c->sel ? 3 * c->numnp_sel : c->neq;
  if(numeq)
    *numeq = c->numeq;
  return ICARAT_OK;
  ICARAT_API_END
}

int icarat_stream(const icarat_ctx *c, void **stream)
{
  ICARAT_API_BEGIN
  IREQUIRE(c && stream, ICARAT_ERR_ARG, "null argument");
  *stream = (void *)c->stream;
  return ICARAT_OK;
  ICARAT_API_END
}

int icarat_synchronize(icarat_ctx *c)
{
  ICARAT_API_BEGIN
  check_ctx(c);
  ICK(cudaStreamSynchronize(c->stream));
  return ICARAT_OK;
  ICARAT_API_END
}

int icarat_dof_map(const icarat_ctx *c, int *node_dof)
{
  ICARAT_API_BEGIN
  IREQUIRE(c && node_dof, ICARAT_ERR_ARG, "null argument");
  if(c->sel)
    for(size_t q = 0; q < c->sel_node_h.size(); q++)
      for(int d = 0; d < 3; d++)
        node_dof[3 * q + d] = c->dof[3 * (size_t)c->sel_node_h[q] + d];
  else
    std::memcpy(node_dof, c->dof.data(), sizeof(int) * c->dof.size());
  return ICARAT_OK;
  ICARAT_API_END
}

int icarat_fext(const icarat_ctx *c, double *fext)
{
  ICARAT_API_BEGIN
  IREQUIRE(c && fext, ICARAT_ERR_ARG, "null argument");
  std::memcpy(fext, c->fext_h.data(), sizeof(double) * c->fext_h.size());
  return ICARAT_OK;
  ICARAT_API_END
}

int icarat_element_stiffness(const icarat_ctx *c, double *ke, double *volume)
{
  ICARAT_API_BEGIN
  IREQUIRE(c, ICARAT_ERR_ARG, "null context");
  if(ke)
    std::memcpy(ke, c->ke0.k, sizeof(double) * 576);
  if(volume)
    *volume = c->vol0;
  return ICARAT_OK;
  ICARAT_API_END
}

int icarat_set_design(icarat_ctx *c, const double *design_s)
{
  ICARAT_API_BEGIN
  check_ctx(c);
  IREQUIRE(design_s, ICARAT_ERR_ARG, "null argument");
  elem_in(c, design_s, true, c->d_rho);
  set_design_device(c, c->d_rho);
  return ICARAT_OK;
  ICARAT_API_END
}

int icarat_set_design_dev(icarat_ctx *c, const double *design_s)
{
  ICARAT_API_BEGIN
  check_ctx(c);
  IREQUIRE(design_s, ICARAT_ERR_ARG, "null argument");
  if(c->sel)
  {
    elem_in(c, design_s, false, c->d_rho);
    design_s = c->d_rho;
  }
  set_design_device(c, design_s);
  return ICARAT_OK;
  ICARAT_API_END
}

static int apply_K_impl(icarat_ctx *c, const double *u, double *y, bool host)
{
  IREQUIRE(c->design_set, ICARAT_ERR_STATE, "set the design first");
  IREQUIRE(u && y, ICARAT_ERR_ARG, "null argument");
  GridDev g{c->nx, c->ny, c->nz, c->NX, c->NY, c->NZ, c->numnp, c->nelx};
  to_full(c, u, c->d_v1, host);
  launch_apply_K(c, g, c->d_E, c->d_fix, c->d_v1, c->d_Ap, nullptr);
  from_full(c, c->d_Ap, y, host);
  return ICARAT_OK;
}

int icarat_apply_K(icarat_ctx *c, const double *u, double *y)
{
  ICARAT_API_BEGIN
  check_ctx(c);
  return apply_K_impl(c, u, y, true);
  ICARAT_API_END
}

int icarat_apply_K_dev(icarat_ctx *c, const double *u, double *y)
{
  ICARAT_API_BEGIN
  check_ctx(c);
  return apply_K_impl(c, u, y, false);
  ICARAT_API_END
}

static void check_tc_err(icarat_ctx *c)
{
  int err = 0;
  ICK(cudaMemcpy(&err, c->d_tc_err, sizeof(int), cudaMemcpyDeviceToHost));
  if(err)
  {
    ICK(cudaMemset(c->d_tc_err, 0, sizeof(int)));
    throw Error{ICARAT_ERR_CUDA, "tensor-core operator: a bounded wait expired"};
  }
}

} // extern "C"

// Runs f with the context's FP64 products forced to the node stencil
// (tc = -1) or to the FP64 tensor cores on every grid they fit (tc = 2).
template <typename F> static int with_fp64_op(icarat_ctx *c, int tc, F f)
{
  const int saved = c->fp64_tc;
  c->fp64_tc = tc;
  try
  {
    const int st = f();
    c->fp64_tc = saved;
    return st;
  }
  catch(...)
  {
    c->fp64_tc = saved;
    throw;
  }
}

extern "C" {

int icarat_apply_K_op(icarat_ctx *c, int op, const double *u, double *y)
{
  ICARAT_API_BEGIN
  check_ctx(c);
  IREQUIRE(op >= ICARAT_OP_FP64 && op <= ICARAT_OP_TC_FP64, ICARAT_ERR_ARG,
           "unknown operator");
  if(op == ICARAT_OP_FP64 || op == ICARAT_OP_TC_FP64)
  {
    GridDev g{c->nx, c->ny, c->nz, c->NX, c->NY, c->NZ, c->numnp, c->nelx};
    IREQUIRE(op == ICARAT_OP_FP64 || dmma_fits(g), ICARAT_ERR_UNSUPPORTED,
             "grid too large for the FP64 tensor-core operator");
    return with_fp64_op(c, op == ICARAT_OP_TC_FP64 ? 2 : -1,
                        [&] { return apply_K_impl(c, u, y, true); });
  }
  IREQUIRE(c->design_set, ICARAT_ERR_STATE, "set the design first");
  IREQUIRE(u && y, ICARAT_ERR_ARG, "null argument");
  mixed_alloc(c);
  to_full(c, u, c->d_v1, true);
  round_f32(c, c->neq, c->d_v1, c->f_p);
  apply_K_lowp(c, op, c->f_p, c->f_Ap);
  widen_f64(c, c->neq, c->f_Ap, c->d_Ap);
  from_full(c, c->d_Ap, y, true);
  check_tc_err(c);
  return ICARAT_OK;
  ICARAT_API_END
}

int icarat_time_operator_op(icarat_ctx *c, int op, int reps, double *ms_per_launch)
{
  ICARAT_API_BEGIN
  check_ctx(c);
  IREQUIRE(op >= ICARAT_OP_FP64 && op <= ICARAT_OP_TC_FP64, ICARAT_ERR_ARG,
           "unknown operator");
  if(op == ICARAT_OP_FP64 || op == ICARAT_OP_TC_FP64)
  {
    GridDev g{c->nx, c->ny, c->nz, c->NX, c->NY, c->NZ, c->numnp, c->nelx};
    IREQUIRE(op == ICARAT_OP_FP64 || dmma_fits(g), ICARAT_ERR_UNSUPPORTED,
             "grid too large for the FP64 tensor-core operator");
    // the tensor-core operator on any grid size it fits (timing only)
    return with_fp64_op(c, op == ICARAT_OP_TC_FP64 ? 2 : -1,
                        [&] { return icarat_time_operator(c, reps, ms_per_launch); });
  }
  IREQUIRE(reps > 0 && ms_per_launch, ICARAT_ERR_ARG, "bad argument");
  IREQUIRE(c->design_set, ICARAT_ERR_STATE, "set the design first");
  mixed_alloc(c);
  round_f32(c, c->neq, c->d_u, c->f_p);
  apply_K_lowp(c, op, c->f_p, c->f_Ap); // warm-up
  *ms_per_launch = time_cold(c, reps, [&] { apply_K_lowp(c, op, c->f_p, c->f_Ap); });
  check_tc_err(c);
  return ICARAT_OK;
  ICARAT_API_END
}

int icarat_solve(icarat_ctx *c, const icarat_solve_opts *opts, double *val,
                 icarat_solve_info *info)
{
  ICARAT_API_BEGIN
  check_ctx(c);
  const icarat_solve_opts &o = opts ? *opts : kDefaultSolve;
  IREQUIRE(c->design_set, ICARAT_ERR_STATE, "set the design first");
  build_rhs(c);
  icarat_solve_info si{};
  int st = solve_full(c, &o, c->d_rhs, c->d_u, &si);
  c->solved = true;
  c->have_u = true;
  c->last_info = si;
  if(info)
    *info = si;
  if(val)
    from_full(c, c->d_u, val, true);
  return st;
  ICARAT_API_END
}

int icarat_solve_rhs(icarat_ctx *c, const icarat_solve_opts *opts, const double *f,
                     double *u, icarat_solve_info *info)
{
  ICARAT_API_BEGIN
  check_ctx(c);
  IREQUIRE(f, ICARAT_ERR_ARG, "null right-hand side");
  const icarat_solve_opts &o = opts ? *opts : kDefaultSolve;
  IREQUIRE(c->design_set, ICARAT_ERR_STATE, "set the design first");
  to_full(c, f, c->d_rhs, true);
  icarat_solve_info si{};
  int st = solve_full(c, &o, c->d_rhs, c->d_u, &si);
  c->solved = true;
  c->have_u = true;
  c->last_info = si;
  if(info)
    *info = si;
  if(u)
    from_full(c, c->d_u, u, true);
  return st;
  ICARAT_API_END
}

int icarat_node_values(icarat_ctx *c, double *node_val)
{
  ICARAT_API_BEGIN
  check_ctx(c);
  IREQUIRE(node_val, ICARAT_ERR_ARG, "null argument");
  IREQUIRE(c->solved, ICARAT_ERR_STATE, "solve first");
  node_values_dev(c, c->d_v1);
  if(c->sel)
  {
    std::vector<double> all((size_t)c->neq);
    d2h(c, all.data(), c->d_v1, c->neq);
    for(size_t q = 0; q < c->sel_node_h.size(); q++)
      for(int d = 0; d < 3; d++)
        node_val[3 * q + d] = all[3 * (size_t)c->sel_node_h[q] + d];
  }
  else
    d2h(c, node_val, c->d_v1, c->neq);
  return ICARAT_OK;
  ICARAT_API_END
}

int icarat_mises(icarat_ctx *c, double *mises)
{
  ICARAT_API_BEGIN
  check_ctx(c);
  IREQUIRE(mises, ICARAT_ERR_ARG, "null argument");
  double *a = stage(c, 0);
  mises_dev(c, a);
  elem_out(c, a, mises, true);
  return ICARAT_OK;
  ICARAT_API_END
}

int icarat_mises_dev(icarat_ctx *c, double *mises)
{
  ICARAT_API_BEGIN
  check_ctx(c);
  IREQUIRE(mises, ICARAT_ERR_ARG, "null argument");
  if(c->sel)
  {
    double *a = stage(c, 0);
    mises_dev(c, a);
    elem_out(c, a, mises, false);
  }
  else
    mises_dev(c, mises);
  return ICARAT_OK;
  ICARAT_API_END
}

int icarat_write_vtk_arrays(const char *path, int binary, int nx, int ny, int nz, double lx,
                            double ly, double lz, const double *node_val,
                            const double *density, const double *mises)
{
  ICARAT_API_BEGIN
  write_vtk(path, binary != 0, nx, ny, nz, lx, ly, lz, node_val, density, mises);
  return ICARAT_OK;
  ICARAT_API_END
}

int icarat_voxelize(int device, const double *tri, int ntri, int nx, int ny, int nz,
                    const double *origin, const double *pitch, unsigned char *mask)
{
  ICARAT_API_BEGIN
  voxelize(device, tri, ntri, nx, ny, nz, origin, pitch, mask);
  return ICARAT_OK;
  ICARAT_API_END
}

int icarat_write_vtk(icarat_ctx *c, const char *path, int binary)
{
  ICARAT_API_BEGIN
  check_ctx(c);
  IREQUIRE(path, ICARAT_ERR_ARG, "null argument");
  no_selection(c, "icarat_write_vtk");
  IREQUIRE(c->solved, ICARAT_ERR_STATE, "solve first");
  std::vector<double> nv((size_t)c->neq), rho((size_t)c->nelx), mis((size_t)c->nelx);
  node_values_dev(c, c->d_v1);
  d2h(c, nv.data(), c->d_v1, c->neq);
  d2h(c, rho.data(), c->d_rho, c->nelx);
  double *a = stage(c, 0);
  mises_dev(c, a);
  d2h(c, mis.data(), a, c->nelx);
  write_vtk(path, binary != 0, c->nx, c->ny, c->nz, c->lx, c->ly, c->lz, nv.data(),
            rho.data(), mis.data());
  return ICARAT_OK;
  ICARAT_API_END
}

int icarat_compliance(icarat_ctx *c, double *compliance)
{
  ICARAT_API_BEGIN
  check_ctx(c);
  IREQUIRE(compliance, ICARAT_ERR_ARG, "null argument");
  IREQUIRE(c->solved, ICARAT_ERR_STATE, "solve first");
  *compliance = compliance_dev(c);
  return ICARAT_OK;
  ICARAT_API_END
}

int icarat_sensitivity(icarat_ctx *c, double scale, double *dfds, double *dgds)
{
  ICARAT_API_BEGIN
  check_ctx(c);
  double *a = stage(c, 0), *b = stage(c, 1);
  sensitivity_dev(c, scale, dfds ? a : nullptr, dgds ? b : nullptr);
  if(dfds)
    elem_out(c, a, dfds, true);
  if(dgds)
    elem_out(c, b, dgds, true);
  return ICARAT_OK;
  ICARAT_API_END
}

int icarat_sensitivity_dev(icarat_ctx *c, double scale, double *dfds, double *dgds)
{
  ICARAT_API_BEGIN
  check_ctx(c);
  if(c->sel)
  {
    double *a = stage(c, 0), *b = stage(c, 1);
    sensitivity_dev(c, scale, dfds ? a : nullptr, dgds ? b : nullptr);
    if(dfds)
      elem_out(c, a, dfds, false);
    if(dgds)
      elem_out(c, b, dgds, false);
  }
  else
    sensitivity_dev(c, scale, dfds, dgds);
  return ICARAT_OK;
  ICARAT_API_END
}

int icarat_filter_setup(icarat_ctx *c, double radius)
{
  ICARAT_API_BEGIN
  check_ctx(c);
  filter_setup(c, radius);
  return ICARAT_OK;
  ICARAT_API_END
}

int icarat_density_filter(icarat_ctx *c, const double *in, double *out, int is_sens)
{
  ICARAT_API_BEGIN
  check_ctx(c);
  IREQUIRE(in && out, ICARAT_ERR_ARG, "null argument");
  double *a = stage(c, 0), *b = stage(c, 1);
  elem_in(c, in, true, a);
  filter_apply(c, a, b, is_sens != 0);
  elem_out(c, b, out, true);
  return ICARAT_OK;
  ICARAT_API_END
}

int icarat_density_filter_dev(icarat_ctx *c, const double *in, double *out,
                              int is_sens)
{
  ICARAT_API_BEGIN
  check_ctx(c);
  IREQUIRE(in && out && in != out, ICARAT_ERR_ARG, "need distinct in/out");
  if(c->sel)
  {
    double *a = stage(c, 0), *b = stage(c, 1);
    elem_in(c, in, false, a);
    filter_apply(c, a, b, is_sens != 0);
    elem_out(c, b, out, false);
  }
  else
    filter_apply(c, in, out, is_sens != 0);
  return ICARAT_OK;
  ICARAT_API_END
}

int icarat_helmholtz_setup(icarat_ctx *c, double radius)
{
  ICARAT_API_BEGIN
  check_ctx(c);
  no_selection(c, "the Helmholtz filter");
  helm_setup(c, radius);
  return ICARAT_OK;
  ICARAT_API_END
}

int icarat_helmholtz_filter(icarat_ctx *c, const double *in, double *out, int is_sens,
                            double rtol, int maxit, icarat_solve_info *info)
{
  ICARAT_API_BEGIN
  check_ctx(c);
  IREQUIRE(in && out, ICARAT_ERR_ARG, "null argument");
  double *a = stage(c, 0), *b = stage(c, 1);
  h2d(c, a, in, c->nelx);
  const int st = helm_filter(c, a, b, is_sens != 0, rtol, maxit, info);
  d2h(c, out, b, c->nelx);
  return st;
  ICARAT_API_END
}

int icarat_helmholtz_filter_dev(icarat_ctx *c, const double *in, double *out, int is_sens,
                                double rtol, int maxit, icarat_solve_info *info)
{
  ICARAT_API_BEGIN
  check_ctx(c);
  IREQUIRE(in && out && in != out, ICARAT_ERR_ARG, "need distinct in/out");
  return helm_filter(c, in, out, is_sens != 0, rtol, maxit, info);
  ICARAT_API_END
}

int icarat_sensitivity_filter(icarat_ctx *c, const double *design_s,
                              const double *dfds, double *out)
{
  ICARAT_API_BEGIN
  check_ctx(c);
  IREQUIRE(design_s && dfds && out, ICARAT_ERR_ARG, "null argument");
  double *a = stage(c, 0), *b = stage(c, 1), *o = stage(c, 2);
  elem_in(c, design_s, true, a);
  elem_in(c, dfds, true, b);
  sensitivity_filter_dev(c, a, b, o);
  elem_out(c, o, out, true);
  return ICARAT_OK;
  ICARAT_API_END
}

static int threshold_impl(icarat_ctx *c, const double *in, double beta, double T,
                          double *out, bool der)
{
  check_ctx(c);
  IREQUIRE(in && out, ICARAT_ERR_ARG, "null argument");
  double *a = stage(c, 0), *b = stage(c, 1);
  elem_in(c, in, true, a);
  threshold_dev(c, a, beta, T, b, der);
  elem_out(c, b, out, true);
  return ICARAT_OK;
}

int icarat_threshold(icarat_ctx *c, const double *in, double beta, double T,
                     double *out)
{
  ICARAT_API_BEGIN
  return threshold_impl(c, in, beta, T, out, false);
  ICARAT_API_END
}

int icarat_threshold_derivative(icarat_ctx *c, const double *in, double beta, double T,
                                double *out)
{
  ICARAT_API_BEGIN
  return threshold_impl(c, in, beta, T, out, true);
  ICARAT_API_END
}

static const icarat_oc_opts kDefaultOc = {0.15, 0.5, 0.0, 1.0e4, 1.0e-5, 100, 0, 1.0, 0.5, 0};

int icarat_oc_update(icarat_ctx *c, double *x, const double *dfdx, double g,
                     const double *dgdx, const double *xmin, const double *xmax,
                     const icarat_oc_opts *opts, int *steps)
{
  ICARAT_API_BEGIN
  check_ctx(c);
  IREQUIRE(x && dfdx && dgdx && xmin && xmax, ICARAT_ERR_ARG, "null argument");
  double *dx = stage(c, 0), *ddf = stage(c, 1), *ddg = stage(c, 2),
         *dmin = stage(c, 3), *dmax = stage(c, 4);
  elem_in(c, x, true, dx);
  elem_in(c, dfdx, true, ddf);
  elem_in(c, dgdx, true, ddg);
  elem_in(c, xmin, true, dmin);
  elem_in(c, xmax, true, dmax);
  int st = oc_update_dev(c, dx, ddf, g, ddg, dmin, dmax, opts ? opts : &kDefaultOc,
                         steps);
  elem_out(c, dx, x, true);
  return st;
  ICARAT_API_END
}

int icarat_oc_update_dev(icarat_ctx *c, double *x, const double *dfdx, double g,
                         const double *dgdx, const double *xmin, const double *xmax,
                         const icarat_oc_opts *opts, int *steps)
{
  ICARAT_API_BEGIN
  check_ctx(c);
  IREQUIRE(x && dfdx && dgdx && xmin && xmax, ICARAT_ERR_ARG, "null argument");
  if(c->sel)
  {
    double *dx = stage(c, 0), *ddf = stage(c, 1), *ddg = stage(c, 2),
           *dmin = stage(c, 3), *dmax = stage(c, 4);
    elem_in(c, x, false, dx);
    elem_in(c, dfdx, false, ddf);
    elem_in(c, dgdx, false, ddg);
    elem_in(c, xmin, false, dmin);
    elem_in(c, xmax, false, dmax);
    const int st = oc_update_dev(c, dx, ddf, g, ddg, dmin, dmax,
                                 opts ? opts : &kDefaultOc, steps);
    elem_out(c, dx, x, false);
    return st;
  }
  return oc_update_dev(c, x, dfdx, g, dgdx, xmin, xmax, opts ? opts : &kDefaultOc,
                       steps);
  ICARAT_API_END
}

int icarat_loop_init(icarat_ctx *c, const icarat_loop_opts *opts, const double *x0)
{
  ICARAT_API_BEGIN
  check_ctx(c);
  IREQUIRE(opts && x0, ICARAT_ERR_ARG, "null argument");
  return loop_init(c, opts, x0);
  ICARAT_API_END
}

int icarat_loop_step(icarat_ctx *c, icarat_step_info *info)
{
  ICARAT_API_BEGIN
  check_ctx(c);
  return loop_step(c, info);
  ICARAT_API_END
}

int icarat_set_load_cases(icarat_ctx *c, int ncases, const double *fext)
{
  ICARAT_API_BEGIN
  check_ctx(c);
  return set_load_cases(c, ncases, fext);
  ICARAT_API_END
}

int icarat_loop_set_domains(icarat_ctx *c, const int *design_ids, int n_design,
                            const int *nondesign_ids, int n_nondesign)
{
  ICARAT_API_BEGIN
  check_ctx(c);
  return loop_set_domains(c, design_ids, n_design, nondesign_ids, n_nondesign);
  ICARAT_API_END
}

int icarat_loop_is_convergence(icarat_ctx *c, double epsilon, double minstep,
                               int *convergence)
{
  ICARAT_API_BEGIN
  check_ctx(c);
  IREQUIRE(convergence, ICARAT_ERR_ARG, "null argument");
  return loop_is_convergence(c, epsilon, minstep, convergence);
  ICARAT_API_END
}

int icarat_loop_save(icarat_ctx *c, const char *path)
{
  ICARAT_API_BEGIN
  check_ctx(c);
  IREQUIRE(path, ICARAT_ERR_ARG, "null path");
  return loop_save(c, path);
  ICARAT_API_END
}

int icarat_loop_load(icarat_ctx *c, const char *path)
{
  ICARAT_API_BEGIN
  check_ctx(c);
  IREQUIRE(path, ICARAT_ERR_ARG, "null path");
  return loop_load(c, path);
  ICARAT_API_END
}

int icarat_loop_get(icarat_ctx *c, int which, double *out)
{
  ICARAT_API_BEGIN
  check_ctx(c);
  IREQUIRE(out, ICARAT_ERR_ARG, "null argument");
  return loop_get(c, which, out);
  ICARAT_API_END
}

} // extern "C"
