// Internal declarations of the sm_100a implementation behind icarat_gpu.h.
//
// Layout in HBM (all contexts):
//   node vectors  : double[3 * numnp], component-major: (node n, component c)
//                   at c * numnp + n (node id = i + j NX + k NX NY, NX =
//                   nx + 1), so a warp's 32 consecutive nodes read 256
//                   contiguous bytes per component; constrained components
//                   always hold 0 (prescribed values live apart);
//   element arrays: double[nelx], element id = i + j nx + k nx ny;
//   "numeq" vectors of the C ABI are gathered / scattered through d_free
//   (equation number -> c * numnp + node).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <exception>
#include <map>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/icarat_gpu.h"

namespace icarat_b200
{

struct Error
{
  int status;
  std::string msg;
};

void set_last_error(const std::string &msg);

// Process-wide count of this library's kernel launches (graph replays count
// their kernel nodes; launches recorded while capturing a graph do not count).
void note_launch(unsigned long long n = 1);
void set_capturing(bool on);

#define ICK(call)                                                               \
  do                                                                            \
  {                                                                             \
    cudaError_t e_ = (call);                                                    \
    if(e_ != cudaSuccess)                                                       \
      throw ::icarat_b200::Error{ICARAT_ERR_CUDA,                               \
                                 std::string(#call) + ": " +                    \
                                     cudaGetErrorString(e_)};                   \
  } while(0)

#define ICARAT_API_BEGIN                                                        \
  try                                                                           \
  {
#define ICARAT_API_END                                                          \
  }                                                                             \
  catch(const ::icarat_b200::Error &e_)                                         \
  {                                                                             \
    ::icarat_b200::set_last_error(e_.msg);                                      \
    return e_.status;                                                           \
  }                                                                             \
  catch(const std::exception &e_)                                               \
  {                                                                             \
    ::icarat_b200::set_last_error(e_.what());                                   \
    return ICARAT_ERR_NOMEM;                                                    \
  }                                                                             \
  catch(...)                                                                    \
  {                                                                             \
    ::icarat_b200::set_last_error("unknown error");                             \
    return ICARAT_ERR_CUDA;                                                     \
  }

#define IREQUIRE(cond, status, msg)                                             \
  do                                                                            \
  {                                                                             \
    if(!(cond))                                                                 \
      throw ::icarat_b200::Error{status, msg};                                  \
  } while(0)

// Programmatic dependent launch.  A kernel launched by launch_chained() may
// be scheduled while the kernel before it in the stream is still draining
// (its launch overlaps the predecessor's tail and completion); every such
// kernel calls chain_wait() before its first global memory access, which
// returns once the predecessor has completed and its writes are visible
// (griddepcontrol.wait, a no-op in a kernel launched without the attribute).
// Nothing triggers dependents early: a dependent is scheduled only after
// every block of its predecessor has exited.
__device__ __forceinline__ void chain_wait()
{
  asm volatile("griddepcontrol.wait;" ::: "memory");
}

// the stop flag of a V-cycle kernel (null: never stop)
__device__ __forceinline__ bool halted(const int *halt)
{
  return halt != nullptr && *halt != 0;
}

template <typename... KArgs, typename... Args>
inline void launch_chained(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem,
                           cudaStream_t st, Args... args)
{
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  ICK(cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...));
}

// Element stiffness (E = 1), passed by value as a kernel parameter: every
// coefficient index is a compile-time constant after unrolling, so the
// 576 entries are read as uniform constant-bank operands.
struct KeParam
{
  double k[576];
};
struct KeParamF
{
  float k[576];
};
// Gauss-averaged stress operator at E = 1 (6 x 24, Voigt rows)
struct StressParam
{
  double s[144];
};

// Structured grid of one level.
struct GridDev
{
  int nx, ny, nz; // elements
  int NX, NY, NZ; // nodes
  int numnp, nelx;
};

// Scalars of a device-resident Krylov loop.
struct CgScalars
{
  double alpha, beta, zr, zr_new, pAp, rr, rnorm, bnorm, tol;
  int iter, maxit, done, status;
  unsigned int counter;
  int pad;
};

// Scalars of the mixed-precision loop (FP32 vectors, FP64 scalars).
struct MxScalars
{
  double alpha, beta, zr, pAp, rr, rr_ref, rr_true, bb, tol2, delta2;
  int iter, maxit, done, status;
  int nstall;   // consecutive refreshes that cut the FP64 residual by < 10 %
  int refresh;  // FP64 residual due after this iteration's update
  int final_;   // iteration cap reached: last refresh, then stop
  int nrefresh; // FP64 residuals evaluated
  int last_refresh; // iteration of the last FP64 residual
  unsigned int counter;
};

// the FP64 residual of the mixed-precision solvers is recomputed at least
// every kRefreshEvery iterations: on ill-conditioned systems (floating solid
// islands in a 1e-9 void) the FP32 recurrence residual can stall while the
// FP32 iterate drifts away from the FP64 solution
constexpr int kRefreshEvery = 50;

// Variants of the tensor-core element-by-element operator (tc_stencil.cu).
enum TcOp
{
  TC_APPLY = 0, // y = K u (constrained rows 0)
  TC_RESID = 1, // y = b - K u (constrained rows 0)
  TC_CHEB = 2,  // d = c1 d + c2 invd (b - K u), y = u + d
  TC_DOT = 3    // y = K u, s->pAp = u . y, s->alpha = s->zr / pAp
};

struct TcArgs
{
  GridDev g;
  const float *E;
  const uint8_t *fix;
  const float *u;
  float *y;
  const uint16_t *keb = nullptr; // [hi, lo][32][32] BF16 bits, row n, column k
  int tiles_x = 0, kc = 0;       // tiles along x; node layers per CTA
  const float *b = nullptr, *invd = nullptr;
  float *d = nullptr;
  float c1 = 0.0f, c2 = 0.0f;
  double *partials = nullptr;
  MxScalars *s = nullptr;
  int *err = nullptr;
  const int *halt = nullptr; // return at entry while *halt != 0
};

// Arguments of the FP64 tensor-core element-by-element operator
// (dmma_stencil.cu); the variants are those of TcOp, with CgScalars.
struct DmArgs
{
  GridDev g;
  KeParam ke;
  const double *E;
  const uint8_t *fix;
  const double *u;
  double *y;
  const double *b = nullptr, *invd = nullptr;
  double *d = nullptr;
  double c1 = 0.0, c2 = 0.0;
  double *partials = nullptr;
  CgScalars *s = nullptr;
  int tiles_x = 0, tiles = 0, kc = 0; // tiles along x, tiles, node layers per CTA
  const int *halt = nullptr;          // return at entry while *halt != 0
};

// Kernel attributes (the dynamic shared-memory limit) and occupancies are per
// device: launch set-up that is done once keeps one slot per device index.
constexpr int kMaxDevices = 64;
inline int device_slot()
{
  int d = 0;
  ICK(cudaGetDevice(&d));
  IREQUIRE(d >= 0 && d < kMaxDevices, ICARAT_ERR_UNSUPPORTED, "device index above 63");
  return d;
}

// Reduction geometry: every grid-stride reduction kernel runs on
// kRedBlocks blocks of kRedThreads threads so that partial sums are summed
// in one fixed order (bit-reproducible on a given GPU).
constexpr int kRedThreads = 256;
constexpr int kMaxRedBlocks = 2048;

// Chebyshev coefficients per Galerkin level (1 / theta, then (c1, c2) of
// steps 1 .. (kGalCoef - 1) / 2)
constexpr int kGalCoef = 16;

struct MgLevel
{
  GridDev g;
  double *E = nullptr;     // nelx, SIMP modulus x 2^level
  uint8_t *fix = nullptr;  // numnp, bit c = component c constrained
  double *invd = nullptr;  // 3 numnp, 1 / diag(K) (0 on constrained)
  double *x = nullptr, *b = nullptr, *r = nullptr, *t = nullptr;
  // FP32 copies of E and invd and FP32 work vectors (mixed-precision solver)
  float *E32 = nullptr, *invd32 = nullptr;
  float *x32 = nullptr, *b32 = nullptr, *r32 = nullptr, *t32 = nullptr;
  // Galerkin coarse operator (levels >= 1 of a Galerkin hierarchy): cell
  // matrices (nelx x 576), node stencil (the 14 blocks o >= 13, 126 x numnp,
  // coefficient-major) and its FP32 copy
  double *Kc = nullptr, *S = nullptr;
  float *S32 = nullptr;
};

struct CoarseSolver
{
  int n = 0;              // free DOFs of the coarsest level
  int bw = 0;             // lower bandwidth of the dense matrix in that order
  int *map = nullptr;     // n -> full index on the coarsest grid
  // two factor buffers (the second only once a lagged set-up needs it):
  double *A[2] = {nullptr, nullptr};    // n x n dense SPD matrix -> its Cholesky factor L
  double *W[2] = {nullptr, nullptr};    // n x n, L^-1
  double *work[2] = {nullptr, nullptr}; // n x n scratch of the inversion, then W^T
  double *vin = nullptr, *vout = nullptr;
  int cur = 0;        // buffer the V-cycle reads
  int pending = -1;   // buffer being factored on the side stream (-1: none)
  bool have = false;  // buffer cur holds the factor of some design
  // per-design set-up graphs: all levels with the factor into buffer b
  // (synchronous), the levels alone, and the factor alone into buffer b
  cudaGraphExec_t setup[2] = {nullptr, nullptr};
  cudaGraphExec_t levels = nullptr;
  cudaGraphExec_t factor[2] = {nullptr, nullptr};
  int setup_kernels = 0, levels_kernels = 0, factor_kernels = 0;
  cudaStream_t side = nullptr;
  cudaEvent_t ev_levels = nullptr, ev_factor[2] = {nullptr, nullptr};
};

struct FilterState
{
  double radius = 0.0;
  int nofs = 0;                 // stencil points
  int rx = 0, ry = 0, rz = 0;   // index reach per axis
  std::vector<int> ofs;         // 3 * nofs (di, dj, dk), ascending element id
  std::vector<double> w;        // nofs weights R - d
  int *d_ofs = nullptr;
  double *d_w = nullptr;
  double *d_aa = nullptr;       // nelx sums of weights (dfilters_ds)
  double *d_ra = nullptr;       // nelx correctly rounded reciprocals 1 / aa
  bool have_forward = false;
};

// Helmholtz PDE filter: element matrix, the 27 x 27 node-class stencil
// table and the CG work vectors (numnp each), allocated by helm_setup
struct HelmState
{
  double radius = 0.0;
  double ke[64] = {}, nj[8] = {}, ns[8] = {};
  double *d_coef = nullptr;
  double *d_invd = nullptr, *d_F = nullptr, *d_val = nullptr, *d_r = nullptr,
         *d_z = nullptr, *d_p = nullptr, *d_Ap = nullptr, *d_partials = nullptr;
  CgScalars *d_cg = nullptr;
  cudaGraphExec_t exec = nullptr; // kHelmChunk iterations
  double *d_oc = nullptr;         // 3 nelx: work of the OC volume functor
  double invd_cls[27] = {};       // Jacobi inverse diagonal per node class
};

struct MmaDev;

struct LoopState
{
  bool init = false;
  icarat_loop_opts opts;
  int optstep = 0;
  double V0 = 0.0;
  // objective of the last step and the one isConvergence last kept
  // (Optimize::object_f / object_old, opt_base.hpp:73-77)
  double object_f = 0.0, object_old = 0.0;
  double *x = nullptr, *xfil = nullptr, *xthr = nullptr, *thrd = nullptr,
         *dfds = nullptr, *dgds = nullptr, *tmp = nullptr, *tmp2 = nullptr,
         *xmin = nullptr, *xmax = nullptr;
  icarat_mma *mma = nullptr;
  // load cases (ncases x neq, node layout) and design domains
  int ncases = 0;
  double *d_cases = nullptr;
  double *d_cases_u = nullptr;      // ncases x neq: each case's last solution
  std::vector<uint8_t> cases_have;  // a case's last solution is held
  double *d_volw = nullptr;   // element volume on design IDs, 0 elsewhere
  uint8_t *d_fixed = nullptr; // 1 on non-design IDs
  // with a selection, the MMA update runs on the kept elements only:
  // x, dfds, dgds, xmin, xmax gathered (5 nelx_sel)
  double *d_sel = nullptr;
};

} // namespace icarat_b200

struct icarat_ctx
{
  int device = 0;
  cudaStream_t stream = nullptr;
  int nx, ny, nz;
  double lx, ly, lz, hx, hy, hz;
  int NX, NY, NZ, numnp, nelx, neq, numeq;
  icarat_material mat;
  icarat_b200::KeParam ke0;
  icarat_b200::KeParamF ke0f; // ke0 rounded to FP32
  icarat_b200::StressParam sb0; // stress operator at E = 1
  double vol0;
  double ke_diag_max; // max_a Ke0[a][a]
  double lam_max_dk;  // bound on lambda_max(D^-1 K) from the element matrix
  int red_blocks;     // reduction grid size
  // host copies
  std::vector<int> dof;        // 3 numnp
  std::vector<double> fext_h;  // numeq
  std::vector<uint8_t> fix_h;  // numnp
  std::vector<double> uD_h;    // 3 numnp prescribed values (0 if free)
  bool has_uD = false;
  // device
  int *d_free = nullptr;
  uint8_t *d_fix = nullptr;
  double *d_uD = nullptr;
  double *d_fext = nullptr;
  double *d_rho = nullptr, *d_E = nullptr;
  float *d_E32 = nullptr; // the moduli rounded to FP32
  double *d_rhs = nullptr, *d_u = nullptr, *d_invd = nullptr;
  double *d_r = nullptr, *d_p = nullptr, *d_z = nullptr, *d_Ap = nullptr;
  double *d_v1 = nullptr, *d_v2 = nullptr; // staging (3 numnp)
  double *d_e1 = nullptr, *d_e2 = nullptr; // staging (nelx)
  double *d_partials = nullptr;            // kMaxRedBlocks * 8
  double *d_scalar = nullptr;              // small scalar results
  double *d_stage = nullptr;               // host-API staging, 6 nelx
  unsigned int *d_counter = nullptr;
  icarat_b200::CgScalars *d_cg = nullptr;
  icarat_b200::CgScalars *h_cg = nullptr; // pinned
  double *h_scalar = nullptr;             // pinned
  // mixed-precision solver (allocated on first use): FP32 iterate x, residual
  // r, preconditioned residual z, direction p and K p
  float *f_x = nullptr, *f_r = nullptr, *f_z = nullptr, *f_p = nullptr, *f_Ap = nullptr;
  icarat_b200::MxScalars *d_mx = nullptr, *h_mx = nullptr;
  // tensor-core operator: Ke0 split into BF16 hi / lo ([2][32][32], padded)
  // and the error flag of its bounded waits
  uint16_t *d_keb = nullptr;
  int *d_tc_err = nullptr;
  int sm_count = 148;
  // operator of the finest level of the FP32 V-cycle (ICARAT_OP_*)
  int mx_fine_op = ICARAT_OP_FP32;
  // FP64 products K u: 0 = by grid size (the FP64 tensor cores on grids of
  // 2M nodes and more, the node stencil below: the measured crossover),
  // 1 = the tensor cores on every grid of 32k nodes and more, 2 = on every
  // grid they fit (explicit operator requests), -1 = the node stencil only
  int fp64_tc = 0;
  // learned preconditioner attached by icarat_ctx_set_net (not owned)
  icarat_net *net = nullptr;
  bool design_set = false, solved = false;
  // d_u holds the solution of an earlier system (kept across design
  // changes): a warm start may begin from it
  bool have_u = false;
  icarat_solve_info last_info{};
  // [mesh] selection (MeshIcarat::modifyMesh): the kept box elements and
  // nodes, numbered in ascending box order; every device array stays in box
  // layout, removed elements have E = 0 and removed nodes are fully fixed
  bool sel = false;
  int nelx_sel = 0, numnp_sel = 0;
  std::vector<int> sel_elem_h, sel_node_h; // kept id -> box id
  uint8_t *d_emask = nullptr;  // box elements: 1 kept (null without selection)
  int *d_sel_elem = nullptr;   // kept element id -> box element id
  double *d_sel_buf = nullptr; // nelx_sel staging of the ABI's element vectors
  // device address of icarat_solve_noalloc's static work buffer on this
  // context's device, resolved when the context is created
  double *noalloc_scratch = nullptr;
  // multigrid
  std::vector<icarat_b200::MgLevel> mg;
  int mg_built_levels = 0;
  // device stop flag of the Krylov iteration whose V-cycles are being
  // enqueued (its scalars' done field; null outside one): the V-cycle
  // kernels return at entry once it is set, so the iterations a graph chunk
  // holds past convergence cost launches only
  const int *mg_halt = nullptr;
  // Galerkin coarse operators: requested by the current solve's options,
  // and built into the hierarchy (which is rebuilt when they differ)
  int mg_galerkin_req = 0, mg_galerkin = 0;
  double *gal_lmax = nullptr; // per level: Chebyshev bound of D^-1 A
  double *gal_coef = nullptr; // per level: kGalCoef Chebyshev coefficients
  double *gal_G = nullptr;    // the 8 child matrices P_s^T Ke0 P_s
  double gal_lam1 = 0.0;      // their Jacobi bound (level 1, unconstrained cells)
  uint8_t *gal_flag1 = nullptr; // level-1 cells with a constrained child node
  int *gal_cells1 = nullptr;    // ... as a list
  int gal_ncells1 = 0;
  icarat_b200::CoarseSolver coarse;
  // filter
  icarat_b200::FilterState filt;
  icarat_b200::HelmState helm;
  // loop
  icarat_b200::LoopState loop;
  // instantiated solver graphs: (method, levels, smooth, chunk, x) -> exec
  std::map<std::tuple<int, int, int, int, const void *>, cudaGraphExec_t> graphs;
  std::map<std::tuple<int, int, int, int, const void *>, int> graph_kernels;
  // right-hand side a graph reads (mixed solver graphs read b at each refresh)
  std::map<std::tuple<int, int, int, int, const void *>, const void *> graph_b;
  unsigned long design_version = 0;
  unsigned long mg_version = ~0ul;
};

namespace icarat_b200
{
// ke0.cpp
void hexa8_stress_operator(double hx, double hy, double hz, double nu, double *s);
void hexa8_stiffness(double hx, double hy, double hz, double nu, double *ke,
                     double *volume);
double jacobi_bound(const double *ke);

// noalloc.cu: resolves c->noalloc_scratch (context creation)
void noalloc_resolve(icarat_ctx *c);

// ctx.cu
// element vectors at the ABI (nelx_sel entries with a selection) <-> box
// layout on the device (removed elements 0)
int abi_nelx(const icarat_ctx *c);
void elem_in(icarat_ctx *c, const double *src, bool host_src, double *d_box);
void elem_out(icarat_ctx *c, const double *d_box, double *dst, bool host_dst);
void to_full(icarat_ctx *c, const double *numeq_in, double *full_out,
             bool host_src);
void from_full(icarat_ctx *c, const double *full_in, double *numeq_out,
               bool host_dst);
void set_design_device(icarat_ctx *c, const double *d_rho);
double *dalloc(size_t n);
void dfree(void *p);

// stiffness.cu
void launch_apply_K(icarat_ctx *c, const GridDev &g, const double *E,
                    const uint8_t *fix, const double *u, double *y,
                    double *dot_partials);
void launch_apply_K_f32(icarat_ctx *c, const GridDev &g, const float *E,
                        const uint8_t *fix, const float *u, float *y);
void launch_diag(icarat_ctx *c, const GridDev &g, const double *E,
                 const uint8_t *fix, double *invd, cudaStream_t st = nullptr);
void launch_residual(icarat_ctx *c, const GridDev &g, const double *E,
                     const uint8_t *fix, const double *b, const double *x,
                     double *r);
void launch_fint(icarat_ctx *c, double *d_out_full);

// reduce helpers (stiffness.cu)
double device_dot(icarat_ctx *c, const double *a, const double *b, int n);

// pcg.cu
void release_graphs(icarat_ctx *c);
int mixed_fp64_finish(icarat_ctx *c, const icarat_solve_opts *o, const double *d_b, double *d_x,
                      icarat_solve_info *info, int st);
int solve_full(icarat_ctx *c, const icarat_solve_opts *o, const double *d_b,
               double *d_x, icarat_solve_info *info);

// net.cu: z = s net(r / s) on ctx's grid and current design
template <typename T>
void net_apply(icarat_net *N, icarat_ctx *c, const T *r, double s, T *z);
// reports (ICARAT_ERR_CUDA) a tensor-core wait of the net that ran out
void net_check(icarat_net *N, cudaStream_t st);

// tc_stencil.cu
void launch_ku_tc(icarat_ctx *c, int op, int terms, TcArgs a, cudaStream_t st);
int pick_layers(long tiles, int NZ, long slots, long max_ctas);
// net_tc.cu: tensor-core forward 3x3x3 convolution of the U-net (BF16 bits)
long conv3_tc_packed_size(int cin, int cout);
void conv3_tc_pack(const uint16_t *W, int cin, int cout, uint16_t *wpk, cudaStream_t st);
void conv3_tc_fwd(int X, int Y, int Z, long V, const uint16_t *x, int cin, const uint16_t *wpk,
                  const float *bias, int cout, uint16_t *y, int *err, cudaStream_t st);
// dmma_stencil.cu
bool dmma_fits(const GridDev &g);
void launch_ku_dmma(icarat_ctx *c, int op, DmArgs a, cudaStream_t st);
// FP64 products of this grid by the FP64 tensor-core operator
bool use_dmma(const icarat_ctx *c, const GridDev &g);

// mixed.cu
struct MixedRun
{
  cudaGraphExec_t exec = nullptr; // chunk of iterations
  int kernels = 0;                // kernel nodes per replay
  long max_chunks = 0, chunks = 0;
  int learned_its = 0;
};
void mixed_begin(icarat_ctx *c, const icarat_solve_opts *o, const double *d_b, double *d_x,
                 MixedRun &run);
bool mixed_poll(icarat_ctx *c, const MixedRun &run);
void mixed_chunk(icarat_ctx *c, MixedRun &run);
int mixed_finish(icarat_ctx *c, const MixedRun &run, icarat_solve_info *info);
int mixed_solve(icarat_ctx *c, const icarat_solve_opts *o, const double *d_b,
                double *d_x, icarat_solve_info *info);
void mixed_alloc(icarat_ctx *c);
void mixed_free(icarat_ctx *c);
// y = K u on the fine grid with one of the reduced-precision operators
// (ICARAT_OP_FP32 / ICARAT_OP_TC_BF16X3 / ICARAT_OP_TC_BF16), FP32 vectors
void apply_K_lowp(icarat_ctx *c, int op, const float *u, float *y);
void round_f32(icarat_ctx *c, long n, const double *in, float *out);
void widen_f64(icarat_ctx *c, long n, const float *in, double *out);

// multigrid.cu
// lag: the V-cycle keeps the coarsest factor of the previous design while
// this design's factor is computed on a side stream (first call after a
// hierarchy change: synchronous)
void mg_setup(icarat_ctx *c, int levels, bool lag = false);
void mg_level_apply(icarat_ctx *c, const icarat_solve_opts *o, int level, const double *x,
                    double *y);
// the context's stream waits for a lagged factorization in flight (so that a
// solve's work, side stream included, ends with the solve)
void mg_join(icarat_ctx *c);
double mg_coarse_check(icarat_ctx *c, int levels, int *n_coarse);
// z = M r by one V-cycle (z null: the result stays in the finest level's x)
void mg_vcycle(icarat_ctx *c, const double *r, double *z, int smooth, bool first_done = false);
void mg_vcycle_f32(icarat_ctx *c, const float *r, float *z, int smooth);
// the context's V-cycle stop flag (icarat_ctx::mg_halt) for one scope
struct HaltScope
{
  icarat_ctx *c;
  const int *prev;
  HaltScope(icarat_ctx *c_, const int *h) : c(c_), prev(c_->mg_halt) { c->mg_halt = h; }
  ~HaltScope() { c->mg_halt = prev; }
  HaltScope(const HaltScope &) = delete;
  HaltScope &operator=(const HaltScope &) = delete;
};
void mg_free(icarat_ctx *c);

// filter.cu
void filter_setup(icarat_ctx *c, double radius);
void filter_apply(icarat_ctx *c, const double *d_in, double *d_out,
                  bool is_sens);
void filter_trans2(icarat_ctx *c, const double *in1, const double *in2, double *out1,
                   double *out2);
void filter_free(icarat_ctx *c);
void threshold_dev(icarat_ctx *c, const double *d_in, double beta, double T,
                   double *d_out, bool derivative);

// helmholtz.cu
void helm_element(double hx, double hy, double hz, double R, double *ke, double *nj,
                  double *ns);
void helm_setup(icarat_ctx *c, double radius);
int helm_filter(icarat_ctx *c, const double *d_in, double *d_out, bool is_sens,
                double rtol, int maxit, icarat_solve_info *info);
void helm_free(icarat_ctx *c);

// sens.cu
void node_values_dev(icarat_ctx *c, double *d_node_val);
void mises_dev(icarat_ctx *c, double *d_mises);

// voxel.cu
void voxelize(int device, const double *tri, int ntri, int nx, int ny, int nz,
              const double *origin, const double *pitch, uint8_t *mask);

// vtk.cu
void write_vtk(const char *path, bool binary, int nx, int ny, int nz, double lx, double ly,
               double lz, const double *node_val, const double *density, const double *mises);
double compliance_dev(icarat_ctx *c);
void sensitivity_dev(icarat_ctx *c, double dgds_scale, double *d_dfds,
                     double *d_dgds);

// oc.cu
int oc_update_dev(icarat_ctx *c, double *x, const double *dfdx, double g,
                  const double *dgdx, const double *xmin, const double *xmax,
                  const icarat_oc_opts *o, int *steps);
int oc_update_helm_dev(icarat_ctx *c, double *x, const double *dfdx, double g,
                       const double *dgdx, const double *xmin, const double *xmax,
                       const icarat_oc_opts *o, int *steps, double *fil, double *thr,
                       const double *vol);

// device reductions shared by several kernels
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double *sh)
{
#pragma unroll
  for(int q = 0; q < NV; q++)
    for(int o = 16; o > 0; o >>= 1)
      v[q] += __shfl_down_sync(0xffffffffu, v[q], o);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int nw = (blockDim.x + 31) >> 5;
  __syncthreads();
  if(lane == 0)
#pragma unroll
    for(int q = 0; q < NV; q++)
      sh[q * 32 + w] = v[q];
  __syncthreads();
  if(w == 0)
  {
#pragma unroll
    for(int q = 0; q < NV; q++)
    {
      v[q] = lane < nw ? sh[q * 32 + lane] : 0.0;
      for(int o = 16; o > 0; o >>= 1)
        v[q] += __shfl_down_sync(0xffffffffu, v[q], o);
    }
  }
}

// Stop test of the CG iterations (ScalingCG, CG.cpp:56-99): count the
// iteration, keep ||r||, stop on NaN, on ||r|| < tol ||b|| or past maxit.
__device__ __forceinline__ void cg_check(CgScalars *s, double rr)
{
  s->iter += 1;
  s->rr = rr;
  s->rnorm = sqrt(rr);
  if(!(rr == rr))
  {
    s->done = 1;
    s->status = ICARAT_ERR_NAN;
  }
  else if(s->rnorm < s->tol * s->bnorm)
  {
    s->done = 1;
    s->status = ICARAT_OK;
  }
  else if(s->iter > s->maxit)
  {
    s->done = 1;
    s->status = ICARAT_WARN_MAXITER;
  }
}

// Called by all threads of every block after thread 0 wrote this block's
// partials.  Returns true in exactly one block (the last to arrive), whose
// threads may then read every block's partials.
__device__ __forceinline__ bool last_block(unsigned int *counter)
{
  __shared__ bool am_last;
  __threadfence();
  __syncthreads();
  if(threadIdx.x == 0)
  {
    unsigned int t = atomicAdd(counter, 1u);
    am_last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if(am_last)
    __threadfence();
  return am_last;
}

// Sum NV partial arrays (layout [q][nparts]) in a fixed order; result in
// thread 0 of the calling block.
template <int NV>
__device__ __forceinline__ void sum_partials(const double *partials, int nparts,
                                             double (&v)[NV], double *sh)
{
#pragma unroll
  for(int q = 0; q < NV; q++)
  {
    double s = 0.0;
    for(int i = threadIdx.x; i < nparts; i += blockDim.x)
      s += __ldcg(partials + q * nparts + i);
    v[q] = s;
  }
  block_sum<NV>(v, sh);
}

} // namespace icarat_b200
