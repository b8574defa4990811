/*
 * icarat_gpu.h -- C ABI of the B200 (sm_100a) implementation of ICARAT's
 * linear-static SIMP topology-optimisation inner loop.
 *
 * Plain C: opaque handles, plain pointers and sizes.  Host pointers are owned
 * by the caller and copied in/out; *_dev variants take device pointers on the
 * context's device and copy nothing.  Every function returns an int status
 * (ICARAT_OK = 0, a positive warning, or a negative error).  One context owns
 * all of its device memory and one CUDA stream; a context is not thread-safe,
 * separate contexts may be used from separate threads.
 *
 * Numbering follows the reference exactly:
 *   node id    = i + j (nx+1) + k (nx+1)(ny+1)        (src/io/mesh_icarat.hpp:468)
 *   element id = i + j nx + k nx ny                   (src/io/mesh_icarat.hpp:486)
 *   equation numbers ("numeq" vectors) = free components, node-major, as
 *   countDOF assigns them (src/io/boundary_condition_base.hpp:35-95).
 */
#ifndef ICARAT_GPU_H
#define ICARAT_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

#define ICARAT_OK 0
#define ICARAT_WARN_MAXITER 1    /* iterative loop stopped at its cap */
#define ICARAT_WARN_STAGNATION 2 /* MIXED_IR: FP64 residual stopped falling */
#define ICARAT_ERR_ARG -1        /* bad argument / size */
#define ICARAT_ERR_CUDA -2       /* CUDA runtime error */
#define ICARAT_ERR_NAN -4        /* non-finite value met in a reduction */
#define ICARAT_ERR_STATE -5      /* call order violated (e.g. transposed filter first) */
#define ICARAT_ERR_FILTER -6     /* filter weight sum < 1e-10 (filter.hpp:130-134) */
#define ICARAT_ERR_UNSUPPORTED -7
#define ICARAT_ERR_NOMEM -8

typedef struct icarat_ctx icarat_ctx;
typedef struct icarat_mma icarat_mma;

/* [mesh] division / length of a hexa8 box (MeshIcarat::setParameter,
   src/io/mesh_icarat.hpp:72-140). */
typedef struct
{
  int nx, ny, nz;
  double lx, ly, lz;
} icarat_grid;

/* [material] young = [E1, E2], poisson, penalty (Elastic::setParameter,
   src/problem/elasticity.cpp:19-33); E(rho) = SIMP (elasticity.hpp:13-17). */
typedef struct
{
  double young_min, young_max;
  double poisson;
  double penalty;
} icarat_material;

/* one [boundary_condition] dirichlet entry: flags, values, [[x0,x1],[y0,y1],
   [z0,z1]] (BCIcarat::input_dirich, boundary_condition_icarat.hpp:73-138) */
typedef struct
{
  int flag[3];
  double val[3];
  double box[3][2];
} icarat_dirichlet;

/* one [boundary_condition] neumann entry (boundary_condition_icarat.hpp:
   213-264): a box degenerate in all three ranges is a point load (val added
   to every node inside, :380-396); any other box is a distributed load, the
   traction val integrated over the face of each element that has 4 nodes
   inside the box (:336-378, SurfaceLoad in boundary_condition_base.cpp:
   16-187, including its face choice: nodes 4-7 select the x-min face). */
typedef struct
{
  double val[3];
  double box[3][2];
} icarat_load;

typedef struct
{
  int n_dirichlet;
  const icarat_dirichlet *dirichlet;
  int n_loads;
  const icarat_load *loads;
} icarat_bc;

enum
{
  ICARAT_SOLVER_JACOBI_PCG = 0, /* "Eigen_CG" / "Scaling_CG" semantics */
  ICARAT_SOLVER_MG_PCG = 1,     /* geometric multigrid preconditioned CG */
  ICARAT_SOLVER_MIXED_IR = 2,   /* FP32 multigrid-PCG iterations refined by FP64
                                   residuals (no reference counterpart); an
                                   FP32 iteration that stalls above rtol or
                                   breaks down is finished by FP64 MG-PCG
                                   (iterations add up) */
  ICARAT_SOLVER_LEARNED_FPCG = 3 /* MIXED_IR with the context's learned net as
                                    initial guess and first preconditioner */
};

typedef struct
{
  int method;    /* ICARAT_SOLVER_* */
  double rtol;   /* stop when ||r|| < rtol ||b||  (solvers.hpp:89: 1e-10) */
  int maxit;     /* iteration cap (solvers.hpp:90: 10000) */
  int mg_levels; /* multigrid levels incl. the finest (MG_PCG, MIXED_IR) */
  int mg_smooth; /* smoothing sweeps per level and direction (MG_PCG, MIXED_IR) */
  int chunk;     /* iterations per host convergence check (0 = default: 4 for
                    MG_PCG and MIXED_IR, 16 for JACOBI_PCG); the iterations of
                    a chunk past convergence return at entry and change nothing */
  double refresh; /* MIXED_IR: recompute the residual in FP64 once the FP32
                     recurrence has fallen by this factor (0 = 1e-2) */
  int fine_op;    /* MIXED_IR: ICARAT_OP_* of the finest-level smoothing and
                     residual in the V-cycle (0 = default) */
  int krylov_op;  /* MIXED_IR: ICARAT_OP_* of K p in the Krylov loop (0 = default) */
  int warm_start; /* start from the solution held by the context (the previous
                     solve, e.g. of the previous design; the loop keeps one per
                     load case) instead of 0; MIXED_IR, and JACOBI_PCG / MG_PCG
                     when the solve writes the context's own solution (icarat_solve,
                     the loop): r0 = b - K x0, same stop test ||r|| < rtol ||b|| */
  int fp64_tc;    /* JACOBI_PCG, MG_PCG: FP64 products K u element by element
                     on the FP64 tensor cores (ICARAT_OP_TC_FP64) or by the
                     node stencil on the CUDA cores: 0 (default) and -1 =
                     the node stencil (the faster of the two at every
                     measured size), 1 = tensor cores on every level of 32k
                     nodes and more.  Also the operator of later
                     icarat_apply_K calls on the context. */
  int coarse_lag; /* MG_PCG, MIXED_IR: 1 = the V-cycle keeps the coarsest-level
                     factor of the previous design while this design's factor
                     is computed on a second stream, overlapped with the solve
                     (factor reuse across design iterations; every solve still
                     meets rtol on the current operator).  The first solve on a
                     new hierarchy factors synchronously. */
  int coarse_op;  /* MG_PCG, MIXED_IR: ICARAT_COARSE_* operators of the coarse
                     multigrid levels (0 = rediscretised) */
} icarat_solve_opts;

enum
{
  /* coarse element moduli = 2 x mean of the 8 children, the fine Ke0 and
     the matrix-free stencil on every level (the default) */
  ICARAT_COARSE_REDISCRETISED = 0,
  /* Galerkin products P^T A P of the masked fine operator, assembled per
     coarse cell and applied as 27-point node stencils; their Chebyshev
     bounds come from the cells.  Keeps the multigrid's convergence on
     solid / void designs at the price of a set-up per design and a
     memory-bound coarse-level stencil.  Not for the batch solver. */
  ICARAT_COARSE_GALERKIN = 1
};

typedef struct
{
  int iterations;
  double rel_residual; /* MIXED_IR: of the last FP64 residual */
  int status;
  int refreshes;       /* MIXED_IR: FP64 residual evaluations */
  int learned_iterations; /* LEARNED_FPCG: iterations preconditioned by the net
                             before the multigrid fallback */
} icarat_solve_info;

/* OC::UpdateVariables parameters (OCSolver.hpp:73-79) and the volume functor
   of the sample drivers: g(x) = sum_i thr(filter(x))_i v_i
   (opt_macro_oc.cpp:153-164), thr only when use_threshold != 0; filter is
   the radius filter of icarat_filter_setup (filter_kind 0) or the Helmholtz
   filter of icarat_helmholtz_setup (1, as opt_macro_oc.cpp:158). */
typedef struct
{
  double move, iota, lambda_min, lambda_max, lambda_eps;
  int maxiter;
  int use_threshold;
  double beta, T;
  int filter_kind;
} icarat_oc_opts;

/* ---- library ---------------------------------------------------------- */
/* 10100: icarat_loop_opts.filter_kind and icarat_oc_opts.filter_kind
   appended (Helmholtz filter); callers built against 10000 headers pass the
   shorter structs and must be rebuilt.  A caller checks
   icarat_version() == ICARAT_ABI_VERSION before passing option structs. */
/* 10200: icarat_loop_is_convergence, icarat_loop_save / _load,
   icarat_ctx_create_selection, icarat_selection_ids and
   icarat_batch_autotune_mg added, and the batch
   method ICARAT_SOLVER_MG_PCG (new functions and values; the 10100 structs
   are unchanged). */
/* 10300: icarat_solve_opts.coarse_op appended (Galerkin coarse operators)
   and icarat_mg_level_apply added;
   the loop options embed it, so loop snapshots are layout version 2.
   Callers built against older headers pass the shorter struct and must be
   rebuilt. */
#define ICARAT_ABI_VERSION 10300
int icarat_version(void);
const char *icarat_status_string(int status);
/* message of the last failed call on this thread */
const char *icarat_last_error(void);

/* ---- context: mesh + BC + device state ----------------------------------
 * Replaces MeshIcarat::setParameter/generate, BCIcarat::input_dirich,
 * makeDOF and input_neumann (mesh_icarat.hpp:72-155,
 * boundary_condition_icarat.hpp:73-148, 213-264) and the LinearAnalysis
 * constructor (src/analysis/linear.hpp:43-52). */
int icarat_ctx_create(const icarat_grid *grid, const icarat_material *mat,
                      const icarat_bc *bc, int device, icarat_ctx **out);
/* [mesh] selection (MeshIcarat::generate -> modifyMesh,
 * src/io/mesh_icarat.hpp:139-155, 636-755): the box of icarat_ctx_create cut
 * down to the union of nsel boxes (x0, x1, y0, y1, z0, z1 each, widened by
 * 1e-7): the nodes inside a box and the elements whose centroid is inside
 * one are kept and renumbered in ascending box order; the boundary
 * conditions see the kept mesh only.  Every element / node quantity of the
 * ABI (sizes, design, filter, sensitivities, DOF map, node values, the
 * loop's vectors and domain IDs) is then in the kept numbering.  A kept
 * element with a removed node (the reference's "error in mesh_icarat") and a
 * kept node without a kept element return ICARAT_ERR_ARG.  Not available on
 * such a context (ICARAT_ERR_UNSUPPORTED): the Helmholtz filter, the VTK
 * writer of the box, the learned preconditioner. */
int icarat_ctx_create_selection(const icarat_grid *grid, const icarat_material *mat,
                                const icarat_bc *bc, int nsel, const double *boxes,
                                int device, icarat_ctx **out);
/* box node id of every kept node (numnp entries) and box element id of every
 * kept element (nelx entries); either may be NULL; the identity without a
 * selection */
int icarat_selection_ids(const icarat_ctx *ctx, int *node_ids, int *elem_ids);
int icarat_ctx_destroy(icarat_ctx *ctx);
/* numnp, nelx, neq (= 3 numnp), numeq; of the kept mesh with a selection */
int icarat_sizes(const icarat_ctx *ctx, int *numnp, int *nelx, int *neq,
                 int *numeq);
/* the context's cudaStream_t, as void* */
int icarat_stream(const icarat_ctx *ctx, void **stream);
int icarat_synchronize(icarat_ctx *ctx);
/* node.dof[0..2] for every node (countDOF, boundary_condition_base.hpp:35-95) */
int icarat_dof_map(const icarat_ctx *ctx, int *node_dof);
/* Force::fext_org (numeq) */
int icarat_fext(const icarat_ctx *ctx, double *fext);
/* E = 1 element stiffness (24x24, row-major, element DOF 3a + c) and volume
   (LinearElastic::makeKeFint, src/problem/elasticity.cpp:211-255) */
int icarat_element_stiffness(const icarat_ctx *ctx, double *ke, double *volume);

/* ---- analysis ------------------------------------------------------------ */
/* element[i].setDesignS(design_s[i]) for every element (nelx values) */
int icarat_set_design(icarat_ctx *ctx, const double *design_s);
int icarat_set_design_dev(icarat_ctx *ctx, const double *design_s);
/* y = K_ff u on free DOFs (numeq vectors): the assembled globalK of
   LinearAnalysis::assemblingK (src/analysis/linear.hpp:117-166) times u,
   applied matrix-free. */
int icarat_apply_K(icarat_ctx *ctx, const double *u, double *y);
int icarat_apply_K_dev(icarat_ctx *ctx, const double *u, double *y);
/* LinearAnalysis::solve (src/analysis/linear.hpp:55-104): rhs = fext - fint
   (fint from prescribed values), solve K u = rhs.  val (numeq) may be NULL;
   the solution stays resident for the calls below. */
int icarat_solve(icarat_ctx *ctx, const icarat_solve_opts *opts, double *val,
                 icarat_solve_info *info);
/* solve K u = f for a given right-hand side (numeq) */
int icarat_solve_rhs(icarat_ctx *ctx, const icarat_solve_opts *opts,
                     const double *f, double *u, icarat_solve_info *info);
/* node.val after divideValIntoNode (analysis_utility.hpp:9-31): numnp x 3,
   prescribed values on constrained DOFs, |v| < 1e-15 -> 0 */
int icarat_node_values(icarat_ctx *ctx, double *node_val);
/* element von Mises stress of the last solve (Elastic::makeMisesStress,
   src/problem/elasticity.cpp:166-207: Gauss-averaged De B u_e of the
   truncated nodal values, sqrt(sigma^T V sigma)); nelx values */
int icarat_mises(icarat_ctx *ctx, double *mises);
int icarat_mises_dev(icarat_ctx *ctx, double *mises);
/* Legacy VTK file of the box as the sample drivers' output()
   (opt_macro_mma_nondesign.cpp:220-242 with src/io/export_vtk.hpp): points,
   hexa8 cells, point vectors "displacement" (node values of the last solve),
   cell scalars "density" (the element design) and "mises".  binary = 0
   writes the reference's ASCII format byte for byte, 1 the same sections as
   legacy BINARY (big-endian float32 / int32). */
int icarat_write_vtk(icarat_ctx *ctx, const char *path, int binary);
/* The same writer on host arrays (no device work): node_val numnp x 3,
   density and mises nelx each; any of the three may be NULL (omitted). */
int icarat_write_vtk_arrays(const char *path, int binary, int nx, int ny, int nz,
                            double lx, double ly, double lz, const double *node_val,
                            const double *density, const double *mises);
/* STL surface -> voxel design domain (the job of scripts/stl_to_vtk_voxel.py,
   vtkSelectEnclosedPoints on the voxel centres): mask[i + nx (j + ny k)] = 1
   when the centre origin + (i+1/2, j+1/2, k+1/2) * pitch lies inside the
   closed surface of ntri triangles (tri: 9 doubles each, three xyz
   vertices), by ray parity along +z on the GPU.  mask is a host array of
   nx ny nz bytes.  More than 256 crossings of one voxel column return
   ICARAT_ERR_UNSUPPORTED. */
int icarat_voxelize(int device, const double *tri, int ntri, int nx, int ny, int nz,
                    const double *origin, const double *pitch, unsigned char *mask);
/* object_f = value.val . fext (opt_macro_oc.cpp:110) of the last solve */
int icarat_compliance(icarat_ctx *ctx, double *compliance);
/* driver sensitivity() (opt_macro_oc.cpp:182-212): dfds = -(dE/E) u_e^T Ke
   u_e, dgds = volume * dgds_scale; either output may be NULL */
int icarat_sensitivity(icarat_ctx *ctx, double dgds_scale, double *dfds,
                       double *dgds);
int icarat_sensitivity_dev(icarat_ctx *ctx, double dgds_scale, double *dfds,
                           double *dgds);

/* ---- density filter (Filter<E,N>, src/optimization/filter.hpp) ---------- */
/* the constructor + preNeighbour (:63-70, :254-297) for radius R */
int icarat_filter_setup(icarat_ctx *ctx, double radius);
/* densityFilter (:107-155): forward, or transposed (is_sens != 0), which
   needs an earlier forward call like the reference */
int icarat_density_filter(icarat_ctx *ctx, const double *in, double *out,
                          int is_sens);
int icarat_density_filter_dev(icarat_ctx *ctx, const double *in, double *out,
                              int is_sens);
/* sensitivityFilter (:77-104) with element volumes of the mesh */
int icarat_sensitivity_filter(icarat_ctx *ctx, const double *design_s,
                              const double *dfds, double *out);
/* threshold / thresholdDerivative (:217-249) */
int icarat_threshold(icarat_ctx *ctx, const double *in, double beta, double T,
                     double *out);
int icarat_threshold_derivative(icarat_ctx *ctx, const double *in, double beta,
                                double T, double *out);

/* ---- Helmholtz PDE filter (FilterHelmholtz<E,N>,
 *      src/optimization/filter_helm.hpp) ------------------------------------
 * setup: the constructor (:67-73) for radius R >= 0.  filter: densityFilter
 * (:75-138) with solvName "Eigen_CG": the nodal system K val = F solved by
 * Jacobi-PCG from zero to ||r|| < rtol ||F|| (rtol <= 0: 1e-10, maxit <= 0:
 * 10000, the Solvers defaults of solvers.hpp:89-90); is_sens != 0 is the
 * sensitivity call (sensFlag).  Returns ICARAT_WARN_MAXITER when the CG
 * stopped at its cap; info (may be NULL) gets the iterations and the final
 * ||r|| / ||F||.  threshold / thresholdDerivative (:140-174) are the same
 * maps as icarat_threshold / icarat_threshold_derivative. */
int icarat_helmholtz_setup(icarat_ctx *ctx, double radius);
int icarat_helmholtz_filter(icarat_ctx *ctx, const double *in, double *out,
                            int is_sens, double rtol, int maxit,
                            icarat_solve_info *info);
int icarat_helmholtz_filter_dev(icarat_ctx *ctx, const double *in, double *out,
                                int is_sens, double rtol, int maxit,
                                icarat_solve_info *info);

/* ---- OC (src/optimization/opt-solver/OCSolver.hpp:21-68) ----------------
 * x is updated in place; g is the reference volume (the driver's V0); the
 * volume functor runs on the GPU with the filter of icarat_filter_setup. */
int icarat_oc_update(icarat_ctx *ctx, double *x, const double *dfdx, double g,
                     const double *dgdx, const double *xmin,
                     const double *xmax, const icarat_oc_opts *opts,
                     int *steps);
int icarat_oc_update_dev(icarat_ctx *ctx, double *x, const double *dfdx,
                         double g, const double *dgdx, const double *xmin,
                         const double *xmax, const icarat_oc_opts *opts,
                         int *steps);

/* ---- MMA (src/optimization/opt-solver/MMASolver.hpp:62-116) -------------
 * MMASolver(n, m, a, c, d) on a device; m <= 8 constraints. */
int icarat_mma_create(int device, int n, int m, double a, double c, double d,
                      icarat_mma **out);
int icarat_mma_destroy(icarat_mma *mma);
int icarat_mma_set_move_limit(icarat_mma *mma, double move);
int icarat_mma_set_asymptotes(icarat_mma *mma, double init, double decrease,
                              double increase);
int icarat_mma_set_oscillation(icarat_mma *mma, double albefa);
/* MMASolver::Update (MMASolver.cpp:66-82); dgdx is n x m row-major */
int icarat_mma_update(icarat_mma *mma, double *x, const double *dfdx,
                      const double *gx, const double *dgdx,
                      const double *xmin, const double *xmax);
int icarat_mma_update_dev(icarat_mma *mma, double *x, const double *dfdx,
                          const double *gx, const double *dgdx,
                          const double *xmin, const double *xmax);
/* outer interior-point loops of the last update ("MMA loop:", :151) */
int icarat_mma_last_loops(const icarat_mma *mma, int *outer, int *newton);

/* ---- one design iteration, device resident --------------------------------
 * The loop body of the sample drivers (opt_macro_oc.cpp:83-172,
 * opt_macro_mma_nondesign.cpp:90-178, opt_mma_Helmholtz.cpp:86-170): filter
 * -> (threshold) -> solve -> compliance/volume -> sensitivity -> filter^T ->
 * OC or MMA update.  filter_kind 0 is the radius Filter (filter.hpp), 1 the
 * Helmholtz PDE filter (filter_helm.hpp, CG to the "Eigen_CG" default 1e-10)
 * that opt_macro_oc.cpp:73-74 and opt_mma_Helmholtz.cpp:70-72 use -- for OC
 * also inside the volume functor of the bisection (:153-164). */
typedef struct
{
  int method;        /* 0 = OC, 1 = MMA */
  int use_threshold; /* beta = min(2^(step/40), 16), T below */
  double T;
  double move;
  double xmin, xmax;
  double filter_radius;
  icarat_solve_opts solve;
  int filter_kind; /* 0 radius filter, 1 Helmholtz PDE filter */
} icarat_loop_opts;

typedef struct
{
  int step;
  double compliance;
  double constraint;
  int cg_iterations;
  double cg_rel_residual;
  int update_steps; /* OC bisection steps or MMA Newton steps */
  int status;
} icarat_step_info;

/* ---- solve without device allocation --------------------------------------
 * No counterpart in the reference.  The Jacobi-PCG solve of
 * icarat_solve_rhs (same kernels: the FP64 node stencil from a zero start)
 * for callers that cannot allocate device memory when they call the solver,
 * e.g. a host application that reserved the whole GPU for its own memory pool
 * at start-up, or a deployment that forbids device allocations after
 * initialisation.  This call allocates nothing: its work vectors live in one
 * static device buffer of the library (about 7.4 MB).  The buffer is
 * committed on a device when the first context of that device is created
 * (icarat_ctx_create resolves its address; under lazy module loading that is
 * when the buffer's module is loaded) and is held until the process exits.
 * f and u are device pointers to numeq vectors (the context's equation
 * numbering); opts may be NULL (rtol 1e-10, maxit 10000) and must select
 * ICARAT_SOLVER_JACOBI_PCG with fp64_tc 0 or -1 and warm_start 0 (other
 * values return ICARAT_ERR_UNSUPPORTED).
 * Limit: 3 (nx+1)(ny+1)(nz+1) <= ICARAT_NOALLOC_MAX_DOFS, larger grids return
 * ICARAT_ERR_ARG.  All calls share the one buffer, which keeps the last
 * call's contents (each call clears what must start at zero): calls that
 * overlap on the GPU -- from two threads, or on two contexts of one device --
 * race. */
#define ICARAT_NOALLOC_MAX_DOFS 131072
int icarat_solve_noalloc(icarat_ctx *ctx, const icarat_solve_opts *opts,
                         const double *f, double *u, icarat_solve_info *info);

/* ---- diagnostics (no reference counterpart) ------------------------------ */
/* number of kernels this library has launched in this process */
int icarat_kernel_launches(unsigned long long *count);
/* average device time of the FP64 stiffness stencil y = K u on the current
   design, over `reps` launches timed with CUDA events on the context's
   stream, each after a 256 MiB write that evicts the L2 (cold caches; the
   call allocates and frees that buffer) */
int icarat_time_operator(icarat_ctx *ctx, int reps, double *ms_per_launch);
/* check of the multigrid's coarsest dense solve on the current design:
   builds the hierarchy of `mg_levels` levels, solves K_c x = b for
   b_i = 1 + (i mod 7) / 7 on the coarsest free unknowns through the dense
   inverse factor and returns ||b - K_c x|| / ||b|| with K_c applied by the
   coarsest level's stencil; *n_coarse (may be NULL): number of unknowns */
int icarat_mg_coarse_check(icarat_ctx *ctx, int mg_levels, double *rel_residual,
                           int *n_coarse);
/* y = A_level x on the current design, host vectors of 3 numnp_level
   entries, component-major (c numnp_level + n): the operator the V-cycle of
   `opts` (mg_levels, coarse_op) applies on that level (level 0 = the fine
   stiffness; constrained rows 0).  Builds the hierarchy as a solve would. */
int icarat_mg_level_apply(icarat_ctx *ctx, const icarat_solve_opts *opts, int level,
                          const double *x, double *y);

/* ---- batched solver (no reference counterpart) ---------------------------
   Many independent designs, of equal or different grid sizes, solved
   together.  Every design is a full context (icarat_batch_ctx returns it for
   the per-design calls: set_design, filter, sensitivity, loop_init, ...);
   icarat_batch_solve runs the Krylov iterations of all designs in ONE
   persistent cooperative launch over a work queue of (design, node tile)
   items, replayed from a CUDA graph: FP32 vectors and K p, Jacobi
   preconditioner, flexible beta, FP64 dot products and per-design FP64
   residual refresh (as ICARAT_SOLVER_MIXED_IR), each design stopping on its
   own FP64 residual.  All designs share the element size and the material. */
typedef struct icarat_batch icarat_batch;

typedef struct
{
  double rtol;       /* per design: ||f - K u|| < rtol ||f|| in FP64 */
  int maxit;         /* iteration cap per design */
  double refresh;    /* FP64 refresh once the FP32 residual fell by this factor
                        (0 = 1e-2) */
  int tile;          /* nodes per work item (0 = autotuned, else 256) */
  int blocks_per_sm; /* persistent CTAs per SM (0 = autotuned, else the
                        occupancy limit) */
  int method;        /* 0 = the persistent Jacobi launch above;
                        ICARAT_SOLVER_MG_PCG = one persistent launch of
                        multigrid-PCG over all designs: every design's own
                        geometric multigrid hierarchy (FP32 Chebyshev-smoothed
                        V-cycle, FP64 dense coarsest solve) applied to all
                        designs phase by phase inside the launch, FP64
                        refresh and stopping test, under a CUDA graph, shape
                        from icarat_batch_autotune_mg;
                        ICARAT_SOLVER_MIXED_IR = every design's own
                        mixed-precision multigrid-PCG (FP32 operator and
                        V-cycle, FP64 refresh and stopping test), the designs
                        interleaved on their own streams as CUDA-graph
                        replays of `chunk` iterations */
  int mg_levels;     /* MG_PCG, MIXED_IR: levels (0 = 4); MIXED_IR: a design
                        whose divisions do not halve that often gets fewer;
                        MG_PCG: the smallest count every design supports
                        (at most 8) */
  int chunk;         /* MIXED_IR: iterations per replay (0 = 4) */
  int warm_start;    /* MG_PCG, MIXED_IR: start from each design's last
                        solution (designs not solved yet start from 0) */
} icarat_batch_opts;

int icarat_batch_create(const icarat_grid *grids, const icarat_bc *bcs, int count,
                        const icarat_material *mat, int device, icarat_batch **out);
int icarat_batch_destroy(icarat_batch *batch);
/* the context of design i (owned by the batch) */
int icarat_batch_ctx(icarat_batch *batch, int i, icarat_ctx **ctx);
/* time the candidate (tile, CTAs per SM) shapes on the current designs and
   keep the fastest for later solves; any output pointer may be NULL */
int icarat_batch_autotune(icarat_batch *batch, int *tile, int *blocks_per_sm,
                          double *ms_per_iteration);
/* the same for the persistent multigrid launch (method ICARAT_SOLVER_MG_PCG)
   with mg_levels levels (0 = 4): the fastest (tile, CTAs per SM) of that
   kernel on the current designs, kept for later MG_PCG solves */
int icarat_batch_autotune_mg(icarat_batch *batch, int mg_levels, int *tile,
                             int *blocks_per_sm, double *ms_per_iteration);
/* K u = f for every design (f from its boundary conditions, u kept in its
   context as after icarat_solve); infos: count entries (may be NULL) */
int icarat_batch_solve(icarat_batch *batch, const icarat_batch_opts *opts,
                       icarat_solve_info *infos);
/* u of design i after icarat_batch_solve (numeq of that design) */
int icarat_batch_solution(icarat_batch *batch, int i, double *u);
/* one design iteration of every design (icarat_loop_init on each context
   first) with the batched solve in place of each loop's own solver */
int icarat_batch_loop_step(icarat_batch *batch, const icarat_batch_opts *opts,
                           icarat_step_info *infos);

/* ---- learned preconditioner (no reference counterpart) -------------------
   A 3-D U-net (4 levels, 16 base channels, BF16 weights and activations,
   FP32 sums) on the node grid: input the residual divided by its L2 norm and
   the node density, output the direction of K^-1 r.  Trained on the GPU
   by this library's own forward and backward kernels (Adam) on samples
   (design rho, load f, solution u) that the plain solver produces.
   ICARAT_SOLVER_LEARNED_FPCG uses the net attached to a context: the net's
   prediction as the initial guess, the net as the preconditioner of a
   flexible PCG while every iteration at least halves the residual, and the
   FP32 multigrid V-cycle from the first iteration that does not (fallback),
   all inside the mixed-precision solver (FP64 residual refresh). */
typedef struct icarat_net icarat_net;
int icarat_net_create(int device, unsigned long long seed, icarat_net **out);
int icarat_net_destroy(icarat_net *net);
int icarat_net_num_params(icarat_net *net, long long *n);
/* FP32 master weights in layer order (W[cout][cin][k^3] then b[cout]) */
int icarat_net_get_params(icarat_net *net, float *w);
int icarat_net_set_params(icarat_net *net, const float *w); /* resets Adam */
/* one step on a sample of ctx's grid (rho: nelx, f and u: numeq): forward,
   loss = 1 - cos^2(net(f / s), u) over free DOFs (s = ||f||; the uses of the
   net do not depend on its output's scale) + 0.01 (|net|^2 - 1)^2 (keeps that
   scale near 1), backward, then Adam with learning
   rate lr (lr = 0: gradients only); *loss is the loss before the update */
int icarat_net_train_step(icarat_net *net, icarat_ctx *ctx, const double *rho,
                          const double *f, const double *u, double lr, double *loss);
/* gradients of the last training step, in the order of the parameters */
int icarat_net_get_grads(icarat_net *net, float *g);
/* s net(f / s) on ctx's current design (numeq in and out): a vector along
   the net's estimate of K^-1 f (its scale is not fitted) */
int icarat_net_infer(icarat_net *net, icarat_ctx *ctx, const double *f, double *u);
/* icarat_net_infer with device pointers (numeq vectors on the context's
   device); enqueued on the context's stream, which it synchronizes once to
   read the norm of f and once at the end to check the net's status */
int icarat_net_infer_dev(icarat_net *net, icarat_ctx *ctx, const double *f, double *u);
/* the net used by ICARAT_SOLVER_LEARNED_FPCG on this context (NULL: none) */
int icarat_ctx_set_net(icarat_ctx *ctx, icarat_net *net);

/* ---- stiffness operators by precision (no reference counterpart) -------- */
enum
{
  ICARAT_OP_FP64 = 0,      /* FP64 node stencil on the CUDA cores */
  ICARAT_OP_FP32 = 1,      /* FP32 node stencil on the CUDA cores */
  ICARAT_OP_TC_BF16X3 = 2, /* element-by-element Ke0 U_e on the tensor cores:
                              BF16 hi/lo split, 3 products, FP32 accumulation */
  ICARAT_OP_TC_BF16 = 3,   /* the same with the single product hi x hi */
  ICARAT_OP_TC_FP64 = 4    /* element-by-element Ke0 U_e on the FP64 tensor cores
                              (DMMA), FP64 throughout */
};
/* y = K u (numeq host vectors) on the current design with operator `op`
   (ICARAT_OP_FP64: the node stencil, whatever the context's default);
   reduced-precision operators round u to FP32 first */
int icarat_apply_K_op(icarat_ctx *ctx, int op, const double *u, double *y);
/* icarat_time_operator for operator `op` (FP32 vectors for ops 1-3) */
int icarat_time_operator_op(icarat_ctx *ctx, int op, int reps, double *ms_per_launch);

int icarat_loop_init(icarat_ctx *ctx, const icarat_loop_opts *opts,
                     const double *x0);
int icarat_loop_step(icarat_ctx *ctx, icarat_step_info *info);
/* which: 0 x, 1 filtered, 2 thresholded, 3 dfds, 4 dgds (nelx each) */
int icarat_loop_get(icarat_ctx *ctx, int which, double *out);
/* Optimize::isConvergence(epsilon, minstep) (src/optimization/opt_base.hpp:28-43)
 * on the loop's objective f, the compliance of the last icarat_loop_step (the
 * sum over the load cases in a multi-load loop): *convergence = 0 when
 * |f_old - f| / f < epsilon and the step count > minstep, else 1 and
 * f_old = f.  f_old starts at 0 at icarat_loop_init (the reference leaves it
 * uninitialised).  The sample drivers call it once per step after the
 * objective (opt_macro_oc.cpp:137, with 1e-5 and 50) and leave the loop
 * after the step in which it returned 0. */
int icarat_loop_is_convergence(icarat_ctx *ctx, double epsilon, double minstep,
                               int *convergence);
/* Checkpoint / resume of the device loop (the reference writes VTK files per
 * step, opt_macro_oc.cpp:214-237, but cannot resume): a binary snapshot of
 * the loop options, step count, V0, the convergence test's objectives, the
 * design, the MMA state (asymptotes, two previous designs, iteration count)
 * and the displacement a warm start begins from.  icarat_loop_load re-creates
 * the loop from it on a context of the same mesh and boundary conditions
 * (ICARAT_ERR_ARG otherwise); load cases and design domains are set again
 * afterwards, as after icarat_loop_init.  Later steps then repeat those of
 * the uninterrupted run (with coarse_lag the first resumed solve factors its
 * own coarse level, so its iteration count may differ). */
int icarat_loop_save(icarat_ctx *ctx, const char *path);
int icarat_loop_load(icarat_ctx *ctx, const char *path);
/* Load cases (the vector<Force> of opt_multi_load.cpp:68-80): fext holds
 * ncases load vectors of numeq entries (the layout of icarat_fext), case
 * after case.  With ncases >= 1 icarat_loop_step solves every case on the
 * same design and sums the compliances and the sensitivities in case order
 * (opt_multi_load.cpp:114-174); ncases = 0 returns to the context's own
 * load.  MMA loops only; batch members take one case. */
int icarat_set_load_cases(icarat_ctx *ctx, int ncases, const double *fext);
/* Design / non-design element IDs of the loop (getDesignNonDesignIDs,
 * src/misc/non_design_domain.hpp:9-53, and its box form in
 * opt_macro_mma_nondesign.cpp:247-317): the volume constraint sums over
 * design_ids (NULL: every element), dfds and dgds are zeroed on
 * nondesign_ids after the transposed filter (:161-166).  Call after
 * icarat_loop_init, which clears them; MMA loops only. */
int icarat_loop_set_domains(icarat_ctx *ctx, const int *design_ids, int n_design,
                            const int *nondesign_ids, int n_nondesign);

#ifdef __cplusplus
}
#endif
#endif /* ICARAT_GPU_H */
