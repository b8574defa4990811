// icarat_solve_noalloc: the Jacobi-PCG solve of icarat_solve_rhs, for callers
// that cannot allocate device memory when they call the solver -- for example
// a host application that reserved the whole GPU for its own memory pool at
// start-up, or a deployment that forbids device allocations after
// initialisation.  Every work vector lives in one file-scope static device
// array of fixed size, so the call performs no cudaMalloc / cudaFree and calls
// no allocating library routine.
//
// The kernels are the ones of the ordinary solve (pcg.cu, stiffness.cu,
// ctx.cu); only the work buffers differ.  Host code cannot use the array's
// name as a device address, so the address is resolved with
// cudaGetSymbolAddress when a context is created (with its device current)
// and kept in the context.  Under lazy module loading that call is what loads
// this file's module and commits the array on the device, so it belongs to
// context creation, which allocates anyway, and not to the solve.
#include "stencil.cuh"

namespace icarat_b200
{
MarchPlan spmv_plan(const icarat_ctx *c, const GridDev &g, int &blocks);
// kernels defined in pcg.cu, stiffness.cu and ctx.cu
__global__ void k_cg_init(int n, const double *__restrict__ b,
                          const double *__restrict__ invd, double *__restrict__ x,
                          double *__restrict__ r, double *__restrict__ z,
                          double *__restrict__ p, double *__restrict__ partials,
                          CgScalars *s, double tol, int maxit, int jacobi);
__global__ void k_cg_spmv(GridDev g, MarchPlan m, KeParam ke, const double *__restrict__ E,
                          const uint8_t *__restrict__ fix, const double *__restrict__ p,
                          double *__restrict__ Ap, double *__restrict__ partials,
                          CgScalars *s);
__global__ void k_cg_update_jacobi(int n, const double *__restrict__ invd,
                                   double *__restrict__ x, double *__restrict__ r,
                                   double *__restrict__ z, const double *__restrict__ p,
                                   const double *__restrict__ Ap,
                                   double *__restrict__ partials, CgScalars *s);
__global__ void k_cg_pupdate(int n, const double *__restrict__ z, double *__restrict__ p,
                             const CgScalars *s);
__global__ void k_inv_diag(GridDev g, KeParam ke, const double *__restrict__ E,
                           const uint8_t *__restrict__ fix, double *__restrict__ invd);
__global__ void k_scatter_free(int numeq, const int *__restrict__ free_idx,
                               const double *__restrict__ in, double *__restrict__ out);
__global__ void k_gather_free(int numeq, const int *__restrict__ free_idx,
                              const double *__restrict__ in, double *__restrict__ out);

// b, x, r, p, z, Ap, 1/diag (node vectors of up to the maximum DOF count),
// reduction partials, and the CG scalars.
constexpr size_t kNaVec = ICARAT_NOALLOC_MAX_DOFS;
constexpr size_t kNaPartials = 2 * (size_t)kMaxRedBlocks;
constexpr size_t kNaScalars = (sizeof(CgScalars) + sizeof(double) - 1) / sizeof(double);
constexpr size_t kNaDoubles = 7 * kNaVec + kNaPartials + kNaScalars;

static __device__ __align__(256) double g_noalloc_scratch[kNaDoubles];

// Device address of the static array on the context's device (current when
// this runs); every context resolves its own, so an address never outlives
// the CUDA context it was taken in.
void noalloc_resolve(icarat_ctx *c)
{
  void *ptr = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
  IREQUIRE(e == cudaSuccess && ptr != nullptr, ICARAT_ERR_CUDA,
           std::string("cudaGetSymbolAddress of the no-allocation solve buffer: ") +
               cudaGetErrorString(e));
  c->noalloc_scratch = static_cast<double *>(ptr);
  // load the kernels the solve launches as well (lazy loading would load
  // each on its first launch, inside the solve)
  const void *kernels[] = {(const void *)k_cg_init,          (const void *)k_cg_spmv,
                           (const void *)k_cg_update_jacobi, (const void *)k_cg_pupdate,
                           (const void *)k_inv_diag,         (const void *)k_scatter_free,
                           (const void *)k_gather_free};
  for(const void *k : kernels)
  {
    cudaFuncAttributes a;
    ICK(cudaFuncGetAttributes(&a, k));
  }
}

static int solve_noalloc(icarat_ctx *c, const icarat_solve_opts *opts, const double *f,
                         double *u, icarat_solve_info *info)
{
  IREQUIRE(c && f && u, ICARAT_ERR_ARG, "null argument");
  ICK(cudaSetDevice(c->device));
  IREQUIRE(c->design_set, ICARAT_ERR_STATE, "set the design first");
  icarat_solve_opts o{ICARAT_SOLVER_JACOBI_PCG, 1.0e-10, 10000, 0, 0, 0};
  if(opts)
    o = *opts;
  IREQUIRE(o.method == ICARAT_SOLVER_JACOBI_PCG, ICARAT_ERR_UNSUPPORTED,
           "icarat_solve_noalloc runs Jacobi-PCG only");
  // the node stencil from a zero start is the only form it runs: the FP64
  // tensor-core operator and warm starts would round differently than asked
  IREQUIRE(o.fp64_tc == 0 || o.fp64_tc == -1, ICARAT_ERR_UNSUPPORTED,
           "icarat_solve_noalloc runs the FP64 node stencil only (fp64_tc 0 or -1)");
  IREQUIRE(o.warm_start == 0, ICARAT_ERR_UNSUPPORTED,
           "icarat_solve_noalloc starts from zero (warm_start 0)");
  IREQUIRE((size_t)c->neq <= kNaVec, ICARAT_ERR_ARG,
           "grid too large for icarat_solve_noalloc: 3*(nx+1)*(ny+1)*(nz+1) = " +
               std::to_string(c->neq) + " DOFs, limit ICARAT_NOALLOC_MAX_DOFS = " +
               std::to_string(kNaVec));
  double *S = c->noalloc_scratch;
  IREQUIRE(S != nullptr, ICARAT_ERR_STATE, "no-allocation buffer not resolved");
  double *b = S, *x = S + kNaVec, *r = S + 2 * kNaVec, *p = S + 3 * kNaVec,
         *z = S + 4 * kNaVec, *Ap = S + 5 * kNaVec, *invd = S + 6 * kNaVec;
  double *partials = S + 7 * kNaVec;
  CgScalars *s = reinterpret_cast<CgScalars *>(partials + kNaPartials);
  const GridDev g{c->nx, c->ny, c->nz, c->NX, c->NY, c->NZ, c->numnp, c->nelx};
  const int n = c->neq;
  const int nb_node = (c->numnp + 255) / 256;
  int nb_spmv;
  const MarchPlan mp = spmv_plan(c, g, nb_spmv);
  // the buffer keeps the previous call's contents: clear the scalars (their
  // reduction counter must start at 0) and the right-hand side (constrained
  // components stay 0); every other vector is written before it is read
  ICK(cudaMemsetAsync(s, 0, sizeof(CgScalars), c->stream));
  ICK(cudaMemsetAsync(b, 0, sizeof(double) * n, c->stream));
  if(c->numeq > 0)
  {
    note_launch(1);
    k_scatter_free<<<(c->numeq + 255) / 256, 256, 0, c->stream>>>(c->numeq, c->d_free, f,
                                                                   b);
  }
  note_launch(2);
  k_inv_diag<<<nb_node, 256, 0, c->stream>>>(g, c->ke0, c->d_E, c->d_fix, invd);
  k_cg_init<<<c->red_blocks, kRedThreads, 0, c->stream>>>(n, b, invd, x, r, z, p,
                                                          partials, s, o.rtol, o.maxit, 1);
  ICK(cudaGetLastError());
  const int chunk = o.chunk > 0 ? o.chunk : 16;
  CgScalars hs{};
  const long max_chunks = (long)(o.maxit + 1 + chunk - 1) / chunk + 1;
  for(long ch = 0; ch < max_chunks; ch++)
  {
    ICK(cudaMemcpyAsync(&hs, s, sizeof(CgScalars), cudaMemcpyDeviceToHost, c->stream));
    ICK(cudaStreamSynchronize(c->stream));
    if(hs.done)
      break;
    for(int k = 0; k < chunk; k++)
    {
      note_launch(3);
      k_cg_spmv<<<nb_spmv, 128, 0, c->stream>>>(g, mp, c->ke0, c->d_E, c->d_fix, p, Ap,
                                                 partials, s);
      k_cg_update_jacobi<<<c->red_blocks, kRedThreads, 0, c->stream>>>(
          n, invd, x, r, z, p, Ap, partials, s);
      k_cg_pupdate<<<c->red_blocks, kRedThreads, 0, c->stream>>>(n, z, p, s);
    }
    ICK(cudaGetLastError());
  }
  if(c->numeq > 0)
  {
    note_launch(1);
    k_gather_free<<<(c->numeq + 255) / 256, 256, 0, c->stream>>>(c->numeq, c->d_free, x,
                                                                  u);
  }
  ICK(cudaGetLastError());
  ICK(cudaMemcpyAsync(&hs, s, sizeof(CgScalars), cudaMemcpyDeviceToHost, c->stream));
  ICK(cudaStreamSynchronize(c->stream));
  const int status = hs.done ? hs.status : ICARAT_WARN_MAXITER;
  if(info)
  {
    info->iterations = hs.iter;
    info->rel_residual = hs.bnorm > 0 ? hs.rnorm / hs.bnorm : 0.0;
    info->status = status;
  }
  return status;
}

} // namespace icarat_b200

extern "C" int icarat_solve_noalloc(icarat_ctx *ctx, const icarat_solve_opts *opts,
                                    const double *f, double *u, icarat_solve_info *info)
{
  ICARAT_API_BEGIN
  return icarat_b200::solve_noalloc(ctx, opts, f, u, info);
  ICARAT_API_END
}
