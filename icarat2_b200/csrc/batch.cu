// Batched solve of many independent designs (no reference counterpart; the
// reference solves one design at a time).
//
// Every design is a full icarat_ctx (mesh, boundary conditions, SIMP moduli,
// FP64 right-hand side and solution live there).  The batch adds one
// cooperative persistent kernel that iterates all designs together.  Work
// is a queue of (design, node tile) items, designs back to back, and each
// CTA takes a contiguous run of items, so designs of different sizes share
// the grid in proportion to their node counts.  Per iteration (grid-wide
// barriers between phases):
//   P1  Ap = K p (FP32 node stencil), per-item partial p . Ap
//   P2  alpha = z.r / p.Ap (design sums of the partials, fixed order);
//       x32 += alpha p, r -= alpha Ap, z = D^-1 r; partials z.r, z.Ap, r.r
//   P3  beta = -z.Ap / p.Ap (flexible); p = z + beta p; the design's first
//       item decides an FP64 refresh (r.r fell by `refresh`, below the target,
//       or the cap) and counts it
//   R   (only when some design asked) x += x32, x32 = 0; r = b - K x in FP64;
//       stop on the FP64 residual (OK / MAXITER / STAGNATION / NAN)
// Vectors are FP32 except the FP64 solution and right-hand side; dot products
// and scalars are FP64.  Designs that stop drop out of the queue; the launch
// ends when none is left or after maxit + 2 iterations.
//
// Tuning: nodes per item and CTAs per SM are picked by timing the candidate
// shapes on the batch itself (icarat_batch_autotune).
#include <cooperative_groups.h>

#include <algorithm>
#include <cmath>

#include "batch.cuh"

namespace cg = cooperative_groups;

namespace icarat_b200
{
int loop_step(icarat_ctx *c, icarat_step_info *info);
double loop_pre(icarat_ctx *c);
int loop_post(icarat_ctx *c, int st, const icarat_solve_info &si, double beta,
              icarat_step_info *info);
void build_rhs(icarat_ctx *c);

__global__ void __launch_bounds__(kBatchThreads, 3) k_batch_pcg(BatchArgs a)
{
  cg::grid_group grid = cg::this_grid();
  __shared__ double sh[4 * 32];
  __shared__ double bc[4];
  const int ipb = (a.nitems + gridDim.x - 1) / gridDim.x;
  const int it0 = min(blockIdx.x * ipb, a.nitems), it1 = min(it0 + ipb, a.nitems);
  const int t = threadIdx.x;
  if(blockIdx.x == 0 && t == 0)
  {
    a.ctl[0] = a.ndes; // nobody reads the control words before the first barrier
    a.ctl[1] = a.ctl[2] = 0;
  }

  // ---- init: x = 0, x32 = 0, r = b, z = D^-1 r, p = z; partials b.b, z.r
  for(int item = it0; item < it1; item++)
  {
    const int d = a.item_design[item];
    const BatchDesign &D = a.des[d];
    const int n0 = (item - D.item0) * a.tile;
    double bb = 0.0, rz = 0.0;
    for(int n = n0 + t; n < min(n0 + a.tile, D.g.numnp); n += blockDim.x)
    {
      const int i = n % D.g.NX, j = (n / D.g.NX) % D.g.NY, k = n / (D.g.NX * D.g.NY);
      double dg[3] = {0.0, 0.0, 0.0};
#pragma unroll
      for(int sz = 0; sz < 2; sz++)
#pragma unroll
        for(int sy = 0; sy < 2; sy++)
#pragma unroll
          for(int sx = 0; sx < 2; sx++)
          {
            const double e = load_E(D.E64, D.g, i - 1 + sx, j - 1 + sy, k - 1 + sz);
            const int la = local_node(1 - sx, 1 - sy, 1 - sz);
#pragma unroll
            for(int c = 0; c < 3; c++)
              dg[c] = fma(e, a.ke.k[(3 * la + c) * 25], dg[c]);
          }
      const unsigned f = D.fix[n];
#pragma unroll
      for(int c = 0; c < 3; c++)
      {
        const long id = (long)c * D.g.numnp + n, o = D.off + id;
        const double bi = D.b[id];
        const float iv = ((f >> c) & 1u) ? 0.0f : (float)(dg[c] != 0.0 ? 1.0 / dg[c] : 1.0);
        const float ri = (float)bi, zi = iv * ri;
        D.x64[id] = 0.0;
        a.x32[o] = 0.0f;
        a.invd[o] = iv;
        a.r[o] = ri;
        a.z[o] = zi;
        a.p[o] = zi;
        bb += bi * bi;
        rz += (double)zi * (double)ri;
      }
    }
    double v[2] = {bb, rz};
    block_sum<2>(v, sh);
    if(t == 0)
    {
      a.part[4L * item + 0] = v[0];
      a.part[4L * item + 1] = v[1];
    }
    __syncthreads();
  }
  grid.sync();
  for(int item = it0; item < it1; item++)
  {
    const int d = a.item_design[item];
    const BatchDesign &D = a.des[d];
    if(item != D.item0)
      continue;
    const double bb = design_sum(a, D, 0, sh, bc);
    const double rz = design_sum(a, D, 1, sh, bc);
    if(t == 0)
    {
      BScal &S = a.s[d];
      S.bb = bb;
      S.rz = rz;
      S.rr_ref = S.rr_true = S.rr_nat = bb;
      S.tol2 = a.tol * a.tol * bb;
      S.delta2 = a.delta * a.delta;
      S.iter = 0;
      S.maxit = a.maxit;
      S.refresh = S.final_ = S.nrefresh = S.nstall = S.last_refresh = 0;
      S.status = ICARAT_OK;
      S.done = 0;
      if(!(bb == bb))
      {
        S.done = 1;
        S.status = ICARAT_ERR_NAN;
      }
      else if(bb == 0.0)
        S.done = 1;
      if(S.done)
        atomicSub(&a.ctl[0], 1);
    }
  }
  grid.sync();

  for(int it = 0; it < a.maxit + 2; it++)
  {
    if(*(volatile int *)&a.ctl[0] <= 0)
      break;
    // ---- P1: Ap = K p, partial p . Ap
    for(int item = it0; item < it1; item++)
    {
      const int d = a.item_design[item];
      if(*(volatile int *)&a.s[d].done)
        continue;
      const BatchDesign &D = a.des[d];
      const int n0 = (item - D.item0) * a.tile;
      double pap = 0.0;
      for(int n = n0 + t; n < min(n0 + a.tile, D.g.numnp); n += blockDim.x)
      {
        float acc[3], uc[3];
        node_Ku<float, KeParamF, true>(D.g, a.kef, D.E32, a.p + D.off, n, acc, uc);
        const unsigned f = D.fix[n];
#pragma unroll
        for(int c = 0; c < 3; c++)
        {
          const float y = ((f >> c) & 1u) ? 0.0f : acc[c];
          a.Ap[D.off + (long)c * D.g.numnp + n] = y;
          pap += (double)uc[c] * (double)y;
        }
      }
      double v[1] = {pap};
      block_sum<1>(v, sh);
      if(t == 0)
        a.part[4L * item] = v[0];
      __syncthreads();
    }
    grid.sync();
    // ---- P2: x32, r, z updates; partials z.r, z.Ap, r.r
    {
      int cached = -1;
      double alpha = 0.0;
      for(int item = it0; item < it1; item++)
      {
        const int d = a.item_design[item];
        if(*(volatile int *)&a.s[d].done)
          continue;
        const BatchDesign &D = a.des[d];
        if(d != cached)
        {
          const double pap = design_sum(a, D, 0, sh, bc);
          alpha = a.s[d].rz / pap;
          cached = d;
        }
        const float al = (float)alpha;
        const int n0 = (item - D.item0) * a.tile;
        const long nv = 3L * D.g.numnp;
        double rz = 0.0, zap = 0.0, rr = 0.0;
        for(int n = n0 + t; n < min(n0 + a.tile, D.g.numnp); n += blockDim.x)
#pragma unroll
          for(int c = 0; c < 3; c++)
          {
            const long o = D.off + (long)c * D.g.numnp + n;
            const float pi = a.p[o], api = a.Ap[o];
            a.x32[o] = fmaf(al, pi, a.x32[o]);
            const float ri = fmaf(-al, api, a.r[o]);
            const float zi = a.invd[o] * ri;
            a.r[o] = ri;
            a.z[o] = zi;
            rz += (double)zi * (double)ri;
            zap += (double)zi * (double)api;
            rr += (double)ri * (double)ri;
          }
        (void)nv;
        double v[3] = {rz, zap, rr};
        block_sum<3>(v, sh);
        if(t == 0)
        {
          a.part[4L * item + 1] = v[0];
          a.part[4L * item + 2] = v[1];
          a.part[4L * item + 3] = v[2];
          if(item == D.item0)
            a.s[d].iter += 1;
        }
        __syncthreads();
      }
    }
    grid.sync();
    // ---- P3: p = z + beta p; refresh decision
    {
      int cached = -1;
      double beta = 0.0;
      for(int item = it0; item < it1; item++)
      {
        const int d = a.item_design[item];
        if(*(volatile int *)&a.s[d].done)
          continue;
        const BatchDesign &D = a.des[d];
        if(d != cached)
        {
          const double pap = design_sum(a, D, 0, sh, bc);
          const double zap = design_sum(a, D, 2, sh, bc);
          beta = -zap / pap;
          cached = d;
          if(item == D.item0)
          {
            const double rz = design_sum(a, D, 1, sh, bc);
            const double rr = design_sum(a, D, 3, sh, bc);
            if(t == 0)
            {
              BScal &S = a.s[d];
              S.rz = rz;
              const bool nan = !(rr == rr) || !(beta == beta);
              S.final_ = (nan || S.iter >= S.maxit) ? 1 : 0;
              S.refresh = (S.final_ || rr < S.tol2 || rr < S.delta2 * S.rr_ref ||
                           S.iter - S.last_refresh >= kRefreshEvery)
                              ? 1
                              : 0;
              if(S.refresh)
                atomicAdd(&a.ctl[1 + (it & 1)], 1);
            }
          }
        }
        const float be = (float)beta;
        const int n0 = (item - D.item0) * a.tile;
        for(int n = n0 + t; n < min(n0 + a.tile, D.g.numnp); n += blockDim.x)
#pragma unroll
          for(int c = 0; c < 3; c++)
          {
            const long o = D.off + (long)c * D.g.numnp + n;
            a.p[o] = fmaf(be, a.p[o], a.z[o]);
          }
      }
      if(blockIdx.x == 0 && t == 0)
        a.ctl[1 + ((it + 1) & 1)] = 0; // the counter of the next iteration
    }
    grid.sync();
    if(*(volatile int *)&a.ctl[1 + (it & 1)] == 0)
      continue;
    // ---- R1: x += x32, x32 = 0 for the designs that refresh
    for(int item = it0; item < it1; item++)
    {
      const int d = a.item_design[item];
      const BScal &S = a.s[d];
      if(*(volatile const int *)&S.done || !*(volatile const int *)&S.refresh)
        continue;
      const BatchDesign &D = a.des[d];
      const int n0 = (item - D.item0) * a.tile;
      for(int n = n0 + t; n < min(n0 + a.tile, D.g.numnp); n += blockDim.x)
#pragma unroll
        for(int c = 0; c < 3; c++)
        {
          const long id = (long)c * D.g.numnp + n;
          D.x64[id] += (double)a.x32[D.off + id];
          a.x32[D.off + id] = 0.0f;
        }
    }
    grid.sync();
    // ---- R2: r = b - K x in FP64, z = D^-1 r; partials r.r, z.r
    for(int item = it0; item < it1; item++)
    {
      const int d = a.item_design[item];
      const BScal &S = a.s[d];
      if(*(volatile const int *)&S.done || !*(volatile const int *)&S.refresh)
        continue;
      const BatchDesign &D = a.des[d];
      const int n0 = (item - D.item0) * a.tile;
      double rr = 0.0, rz = 0.0;
      for(int n = n0 + t; n < min(n0 + a.tile, D.g.numnp); n += blockDim.x)
      {
        double acc[3];
        node_Ku_lean(D.g, a.ke, D.E64, D.x64, n, acc);
        const unsigned f = D.fix[n];
#pragma unroll
        for(int c = 0; c < 3; c++)
        {
          const long id = (long)c * D.g.numnp + n, o = D.off + id;
          const double ri = ((f >> c) & 1u) ? 0.0 : D.b[id] - acc[c];
          const float r32 = (float)ri, zi = a.invd[o] * r32;
          a.r[o] = r32;
          a.z[o] = zi;
          rr += ri * ri;
          rz += (double)zi * (double)r32;
        }
      }
      double v[2] = {rr, rz};
      block_sum<2>(v, sh);
      if(t == 0)
      {
        a.part[4L * item + 0] = v[0];
        a.part[4L * item + 1] = v[1];
      }
      __syncthreads();
    }
    grid.sync();
    // ---- R3: stop test on the FP64 residual
    for(int item = it0; item < it1; item++)
    {
      const int d = a.item_design[item];
      const BatchDesign &D = a.des[d];
      if(item != D.item0)
        continue;
      BScal &S = a.s[d];
      if(*(volatile int *)&S.done || !*(volatile int *)&S.refresh)
        continue;
      const double rr = design_sum(a, D, 0, sh, bc);
      const double rz = design_sum(a, D, 1, sh, bc);
      if(t == 0)
      {
        S.nstall = rr > 0.81 * S.rr_true ? S.nstall + 1 : 0;
        S.rr_true = S.rr_ref = rr;
        S.rz = rz;
        S.nrefresh += 1;
        S.last_refresh = S.iter;
        S.refresh = 0;
        if(!(rr == rr))
        {
          S.done = 1;
          S.status = ICARAT_ERR_NAN;
        }
        else if(rr < S.tol2)
        {
          S.done = 1;
          S.status = ICARAT_OK;
        }
        else if(S.final_)
        {
          S.done = 1;
          S.status = ICARAT_WARN_MAXITER;
        }
        else if(S.nstall >= 3)
        {
          S.done = 1;
          S.status = ICARAT_WARN_STAGNATION;
        }
        if(S.done)
          atomicSub(&a.ctl[0], 1);
      }
    }
    grid.sync();
  }
}

} // namespace icarat_b200

using namespace icarat_b200;

struct icarat_batch
{
  int device = 0;
  cudaStream_t stream = nullptr;
  std::vector<icarat_ctx *> ctx;
  KeParam ke;
  KeParamF kef;
  long total_nv = 0; // FP32 node-vector length of all designs
  float *buf = nullptr; // x32, r, z, p, Ap, invd back to back
  BatchDesign *d_des = nullptr;
  int *d_item_design = nullptr;
  double *d_part = nullptr;
  BScal *d_s = nullptr, *h_s = nullptr;
  int *d_ctl = nullptr;
  int nitems = 0, items_tile = 0; // items built for this tile
  int tile = 0, blocks_per_sm = 0; // tuned shape (0 = not tuned)
  int occ = 0;                     // co-resident CTAs per SM
  cudaGraphExec_t graph = nullptr;
  std::tuple<int, int, double, int, double> graph_key{};
  std::vector<cudaEvent_t> ev;
  cudaEvent_t done_ev = nullptr;
  // persistent multigrid launch (method ICARAT_SOLVER_MG_PCG)
  BmDesign *d_bm = nullptr;
  std::vector<BmDesign> h_bm;
  int *d_lv_items[kBmMaxLevels] = {};
  int lv_nitems[kBmMaxLevels] = {};
  int *d_citems = nullptr;
  int c_nitems = 0;
  int *d_lv_col[kBmMaxLevels] = {};
  int lv_col_items[kBmMaxLevels] = {};
  double *d_partc = nullptr;
  double *d_y = nullptr;
  int mg_levels = 0, mg_tile = 0;         // tables built for these
  int occ_mg = 0;                         // co-resident CTAs per SM
  int mg_tuned_tile = 0, mg_tuned_bpsm = 0; // icarat_batch_autotune_mg
  cudaGraphExec_t mg_graph = nullptr;
  std::tuple<int, int, double, int, double, int, int> mg_key{};
};

int icarat_ctx_create_impl(const icarat_grid *grid, const icarat_material *mat,
                           const icarat_bc *bc, int device, icarat_ctx **out);

static void batch_items(icarat_batch *B, int tile)
{
  if(B->items_tile == tile)
    return;
  ICK(cudaStreamSynchronize(B->stream)); // launches in flight read the old tables
  std::vector<BatchDesign> des(B->ctx.size());
  std::vector<int> item_design;
  long off = 0;
  for(size_t d = 0; d < B->ctx.size(); d++)
  {
    icarat_ctx *c = B->ctx[d];
    BatchDesign &D = des[d];
    D.g = GridDev{c->nx, c->ny, c->nz, c->NX, c->NY, c->NZ, c->numnp, c->nelx};
    D.E32 = c->d_E32;
    D.E64 = c->d_E;
    D.fix = c->d_fix;
    D.b = c->d_rhs;
    D.x64 = c->d_u;
    D.off = off;
    D.item0 = (int)item_design.size();
    D.nitems = (c->numnp + tile - 1) / tile;
    for(int i = 0; i < D.nitems; i++)
      item_design.push_back((int)d);
    off += 3L * c->numnp;
  }
  dfree(B->d_item_design);
  dfree(B->d_part);
  B->d_item_design = nullptr;
  B->d_part = nullptr;
  B->nitems = (int)item_design.size();
  ICK(cudaMalloc(&B->d_item_design, sizeof(int) * item_design.size()));
  ICK(cudaMemcpy(B->d_item_design, item_design.data(), sizeof(int) * item_design.size(),
                 cudaMemcpyHostToDevice));
  B->d_part = dalloc(4 * item_design.size());
  ICK(cudaMemcpy(B->d_des, des.data(), sizeof(BatchDesign) * des.size(),
                 cudaMemcpyHostToDevice));
  B->items_tile = tile;
  if(B->graph)
  {
    cudaGraphExecDestroy(B->graph);
    B->graph = nullptr;
  }
  // the multigrid launch's graph and tables hold the old item table too
  if(B->mg_graph)
  {
    cudaGraphExecDestroy(B->mg_graph);
    B->mg_graph = nullptr;
  }
  B->mg_levels = B->mg_tile = 0;
}

// Right-hand sides of every design, and the batch stream ordered after
// everything already queued on the design streams.
static void batch_prepare(icarat_batch *B, bool rhs)
{
  for(size_t d = 0; d < B->ctx.size(); d++)
  {
    icarat_ctx *c = B->ctx[d];
    IREQUIRE(c->design_set, ICARAT_ERR_STATE, "set the design of every batch member first");
    if(rhs)
      build_rhs(c);
    ICK(cudaEventRecord(B->ev[d], c->stream));
    ICK(cudaStreamWaitEvent(B->stream, B->ev[d], 0));
  }
}

static void batch_launch(icarat_batch *B, int tile, int bpsm, double rtol, int maxit,
                         double refresh)
{
  batch_items(B, tile);
  BatchArgs a;
  a.ke = B->ke;
  a.kef = B->kef;
  a.des = B->d_des;
  a.ndes = (int)B->ctx.size();
  a.item_design = B->d_item_design;
  a.nitems = B->nitems;
  a.tile = tile;
  const long nv = B->total_nv;
  a.x32 = B->buf;
  a.r = B->buf + nv;
  a.z = B->buf + 2 * nv;
  a.p = B->buf + 3 * nv;
  a.Ap = B->buf + 4 * nv;
  a.invd = B->buf + 5 * nv;
  a.part = B->d_part;
  a.s = B->d_s;
  a.ctl = B->d_ctl;
  a.maxit = maxit;
  a.tol = rtol;
  a.delta = refresh;
  const int sms = B->ctx[0]->sm_count;
  const int blocks = sms * std::max(1, std::min(bpsm, B->occ));
  void *args[] = {&a};
  note_launch();
  ICK(cudaLaunchCooperativeKernel((void *)k_batch_pcg, dim3(blocks), dim3(kBatchThreads), args,
                                  0, B->stream));
}

// The solve as a CUDA graph (one graph per shape and options).
static void batch_run(icarat_batch *B, int tile, int bpsm, double rtol, int maxit,
                      double refresh)
{
  const auto key = std::make_tuple(tile, bpsm, rtol, maxit, refresh);
  if(!B->graph || B->graph_key != key)
  {
    if(B->graph)
    {
      cudaGraphExecDestroy(B->graph);
      B->graph = nullptr;
    }
    batch_items(B, tile);
    cudaGraph_t g;
    ICK(cudaStreamBeginCapture(B->stream, cudaStreamCaptureModeThreadLocal));
    set_capturing(true);
    try
    {
      batch_launch(B, tile, bpsm, rtol, maxit, refresh);
    }
    catch(...)
    {
      set_capturing(false);
      cudaStreamEndCapture(B->stream, &g);
      throw;
    }
    set_capturing(false);
    ICK(cudaStreamEndCapture(B->stream, &g));
    ICK(cudaGraphInstantiate(&B->graph, g, 0));
    cudaGraphDestroy(g);
    B->graph_key = key;
  }
  ICK(cudaGraphLaunch(B->graph, B->stream));
  note_launch();
}

static int pick_tile(icarat_batch *B, const icarat_batch_opts *o)
{
  if(o && o->tile > 0)
    return o->tile;
  return B->tile > 0 ? B->tile : 256;
}

static int pick_bpsm(icarat_batch *B, const icarat_batch_opts *o)
{
  if(o && o->blocks_per_sm > 0)
    return std::min(o->blocks_per_sm, B->occ);
  return B->blocks_per_sm > 0 ? B->blocks_per_sm : B->occ;
}

// Largest level count <= want (at least 2) for which every division of the
// design halves level-1 times.
static int design_levels(const icarat_ctx *c, int want)
{
  int L = std::max(2, want);
  while(L > 2)
  {
    const int m = 1 << (L - 1);
    if(c->nx % m == 0 && c->ny % m == 0 && c->nz % m == 0)
      break;
    L--;
  }
  return L;
}

static void note_result(icarat_ctx *c, const icarat_solve_info &si, icarat_solve_info *out,
                        int &worst)
{
  c->solved = true;
  c->have_u = true;
  c->last_info = si;
  if(out)
    *out = si;
  if(si.status < 0)
    worst = std::min(worst, si.status);
  else if(worst >= 0 && si.status > worst)
    worst = si.status;
}

// Every design's own mixed-precision multigrid-PCG (the solver of
// ICARAT_SOLVER_MIXED_IR with the FP32 operator on every level), the
// designs interleaved: each round queues one graph replay of `chunk`
// iterations on the stream of every design still running, then waits for
// the designs one by one, so that while the host reads one design's stop
// flag the others' replays run on the GPU.  The multigrid set-ups
// (transfer of the moduli, coarse dense factor) are queued on the design
// streams too and overlap in the same way.
static int batch_solve_concurrent(icarat_batch *B, const icarat_batch_opts *o, double rtol,
                                  int maxit, double refresh, icarat_solve_info *infos)
{
  const size_t n = B->ctx.size();
  const int want = o->mg_levels > 0 ? o->mg_levels : 4;
  IREQUIRE(want >= 2 && want <= 12, ICARAT_ERR_ARG, "mg_levels must be in [2, 12]");
  IREQUIRE(o->chunk >= 0, ICARAT_ERR_ARG, "chunk must be non-negative");
  std::vector<MixedRun> run(n);
  std::vector<icarat_solve_opts> opts(n);
  for(size_t d = 0; d < n; d++)
  {
    icarat_ctx *c = B->ctx[d];
    icarat_solve_opts &so = opts[d];
    so = icarat_solve_opts{};
    so.method = ICARAT_SOLVER_MIXED_IR;
    so.rtol = rtol;
    so.maxit = maxit;
    so.mg_levels = design_levels(c, want);
    so.chunk = o->chunk;
    so.refresh = refresh;
    so.fine_op = ICARAT_OP_FP32;
    so.krylov_op = ICARAT_OP_FP32;
    so.warm_start = (o->warm_start && c->have_u) ? 1 : 0;
    mixed_begin(c, &so, c->d_rhs, c->d_u, run[d]);
    ICK(cudaEventRecord(B->ev[d], c->stream));
  }
  std::vector<char> active(n, 1);
  for(size_t live = n; live > 0;)
  {
    live = 0;
    for(size_t d = 0; d < n; d++)
    {
      if(!active[d])
        continue;
      icarat_ctx *c = B->ctx[d];
      ICK(cudaEventSynchronize(B->ev[d]));
      if(!mixed_poll(c, run[d]))
      {
        active[d] = 0;
        continue;
      }
      mixed_chunk(c, run[d]);
      ICK(cudaEventRecord(B->ev[d], c->stream));
      live++;
    }
  }
  int worst = ICARAT_OK;
  for(size_t d = 0; d < n; d++)
  {
    icarat_solve_info si{};
    icarat_ctx *c = B->ctx[d];
    // a design whose FP32 iteration stalled or broke down is finished in
    // FP64, as the single-design mixed solve does
    mixed_fp64_finish(c, &opts[d], c->d_rhs, c->d_u, &si, mixed_finish(c, run[d], &si));
    note_result(c, si, infos ? &infos[d] : nullptr, worst);
  }
  return worst;
}

// ---------------------------------------------------------------- multigrid
constexpr int kBmCoarseRows = 8; // coarse dense rows per work item
constexpr int kBmDeg = 2;         // Chebyshev steps per level and direction
constexpr int kBmLayers = 8;      // node layers per column item of the stencil phases

// Item tables of the persistent multigrid launch: node tiles of every level
// of every design, and row blocks of every design's coarsest dense solve.
// Level 0 uses the batch's own item table (batch_items).
static void batch_mg_tables(icarat_batch *B, int L, int tile)
{
  batch_items(B, tile);
  const size_t n = B->ctx.size();
  B->h_bm.assign(n, BmDesign{});
  std::vector<std::vector<int>> lv(L), lvc(L);
  std::vector<int> citems;
  long ylen = 0;
  for(size_t d = 0; d < n; d++)
  {
    icarat_ctx *c = B->ctx[d];
    BmDesign &M = B->h_bm[d];
    for(int l = 0; l < L; l++)
    {
      const GridDev &g = c->mg[l].g;
      BmLevel &V = M.lv[l];
      V.g = g;
      V.item0 = (int)lv[l].size();
      V.nitems = (g.numnp + tile - 1) / tile;
      for(int i = 0; i < V.nitems; i++)
        lv[l].push_back((int)d);
      // stencil phases: blocks of kBatchThreads node columns x chunks of
      // about kBmLayers node layers (balanced: chunk lengths differ by at
      // most one, so that no item is a short remainder)
      V.ncb = (g.NX * g.NY + kBatchThreads - 1) / kBatchThreads;
      {
        const int nch = (g.NZ + kBmLayers - 1) / kBmLayers;
        V.kc = (g.NZ + nch - 1) / nch;
      }
      V.mitem0 = (int)lvc[l].size();
      V.mitems = V.ncb * ((g.NZ + V.kc - 1) / V.kc);
      for(int i = 0; i < V.mitems; i++)
        lvc[l].push_back((int)d);
    }
    M.nc = c->coarse.n;
    M.citem0 = (int)citems.size();
    M.citems = std::max(1, (M.nc + kBmCoarseRows - 1) / kBmCoarseRows);
    for(int i = 0; i < M.citems; i++)
      citems.push_back((int)d);
    ylen += 2L * std::max(1, M.nc);
  }
  if(B->mg_levels != L || B->mg_tile != tile)
  {
    for(int l = 0; l < kBmMaxLevels; l++)
    {
      if(l > 0)
        dfree(B->d_lv_items[l]);
      B->d_lv_items[l] = nullptr;
      B->lv_nitems[l] = 0;
      dfree(B->d_lv_col[l]);
      B->d_lv_col[l] = nullptr;
      B->lv_col_items[l] = 0;
    }
    dfree(B->d_citems);
    dfree(B->d_y);
    dfree(B->d_partc);
    for(int l = 0; l < L; l++)
    {
      ICK(cudaMalloc(&B->d_lv_col[l], sizeof(int) * lvc[l].size()));
      ICK(cudaMemcpy(B->d_lv_col[l], lvc[l].data(), sizeof(int) * lvc[l].size(),
                     cudaMemcpyHostToDevice));
      B->lv_col_items[l] = (int)lvc[l].size();
    }
    B->d_partc = dalloc(4 * lvc[0].size());
    B->d_lv_items[0] = B->d_item_design;
    B->lv_nitems[0] = B->nitems;
    for(int l = 1; l < L; l++)
    {
      ICK(cudaMalloc(&B->d_lv_items[l], sizeof(int) * lv[l].size()));
      ICK(cudaMemcpy(B->d_lv_items[l], lv[l].data(), sizeof(int) * lv[l].size(),
                     cudaMemcpyHostToDevice));
      B->lv_nitems[l] = (int)lv[l].size();
    }
    ICK(cudaMalloc(&B->d_citems, sizeof(int) * citems.size()));
    ICK(cudaMemcpy(B->d_citems, citems.data(), sizeof(int) * citems.size(),
                   cudaMemcpyHostToDevice));
    B->c_nitems = (int)citems.size();
    B->d_y = dalloc(ylen);
    B->mg_levels = L;
    B->mg_tile = tile;
    if(B->mg_graph)
    {
      cudaGraphExecDestroy(B->mg_graph);
      B->mg_graph = nullptr;
    }
  }
  B->d_lv_items[0] = B->d_item_design; // batch_items may have rebuilt it
  // per-design pointers (levels and factor buffers of the contexts) and the
  // Chebyshev coefficients of the smoother (the sequence of smooth() in
  // multigrid.cu)
  long yoff = 0;
  for(size_t d = 0; d < n; d++)
  {
    icarat_ctx *c = B->ctx[d];
    BmDesign &M = B->h_bm[d];
    for(int l = 0; l < L; l++)
    {
      MgLevel &G = c->mg[l];
      BmLevel &V = M.lv[l];
      V.E32 = G.E32;
      V.invd = G.invd32;
      V.fix = G.fix;
      V.x = G.x32;
      V.t = G.t32;
      V.r = G.r32;
      V.b = G.b32;
    }
    M.W = c->coarse.W[c->coarse.cur];
    M.WT = c->coarse.work[c->coarse.cur];
    M.map = c->coarse.map;
    M.cmap = c->coarse.map + M.nc;
    M.v = B->d_y + yoff;
    M.y = M.v + std::max(1, M.nc);
    yoff += 2L * std::max(1, M.nc);
    const double lmax = c->lam_max_dk, lmin = 0.1 * lmax;
    const double theta = 0.5 * (lmax + lmin), delta = 0.5 * (lmax - lmin);
    const double sigma = theta / delta;
    M.inv_theta = (float)(1.0 / theta);
    double rho_old = 1.0 / sigma;
    M.pre_c1[0] = 0.0f;
    M.pre_c2[0] = (float)(1.0 / theta);
    for(int k = 1; k < kBmMaxDeg; k++)
    {
      const double rho = 1.0 / (2.0 * sigma - rho_old);
      M.pre_c1[k] = (float)(rho * rho_old);
      M.pre_c2[k] = (float)(2.0 * rho / delta);
      rho_old = rho;
    }
    for(int k = 0; k < kBmMaxDeg; k++)
    {
      M.post_c1[k] = M.pre_c1[k];
      M.post_c2[k] = M.pre_c2[k];
    }
  }
  if(!B->d_bm)
    ICK(cudaMalloc(&B->d_bm, sizeof(BmDesign) * n));
  ICK(cudaStreamSynchronize(B->stream)); // no launch in flight reads the table
  ICK(cudaMemcpy(B->d_bm, B->h_bm.data(), sizeof(BmDesign) * n, cudaMemcpyHostToDevice));
}

static void batch_mg_launch(icarat_batch *B, int tile, int bpsm, double rtol, int maxit,
                            double refresh, int L, int warm)
{
  BatchArgs a;
  a.ke = B->ke;
  a.kef = B->kef;
  a.des = B->d_des;
  a.ndes = (int)B->ctx.size();
  a.item_design = B->d_item_design;
  a.nitems = B->nitems;
  a.tile = tile;
  const long nv = B->total_nv;
  a.x32 = B->buf;
  a.r = B->buf + nv;
  a.z = B->buf + 2 * nv;
  a.p = B->buf + 3 * nv;
  a.Ap = B->buf + 4 * nv;
  a.invd = B->buf + 5 * nv;
  a.part = B->d_part;
  a.s = B->d_s;
  a.ctl = B->d_ctl;
  a.maxit = maxit;
  a.tol = rtol;
  a.delta = refresh;
  BmArgs m;
  m.levels = L;
  m.deg = kBmDeg;
  m.ctile = kBmCoarseRows;
  m.warm = warm;
  m.bm = B->d_bm;
  for(int l = 0; l < kBmMaxLevels; l++)
  {
    m.lv_item_design[l] = B->d_lv_items[l];
    m.lv_nitems[l] = B->lv_nitems[l];
  }
  m.c_item_design = B->d_citems;
  m.c_nitems = B->c_nitems;
  for(int l = 0; l < kBmMaxLevels; l++)
  {
    m.lv_col_design[l] = B->d_lv_col[l];
    m.lv_col_items[l] = B->lv_col_items[l];
  }
  m.partc = B->d_partc;
  const int sms = B->ctx[0]->sm_count;
  const int blocks = sms * std::max(1, std::min(bpsm, B->occ_mg));
  void *args[] = {&a, &m};
  note_launch();
  ICK(cudaLaunchCooperativeKernel((void *)k_batch_mg, dim3(blocks), dim3(kBatchThreads), args,
                                  0, B->stream));
}

// The multigrid launch as a CUDA graph (one graph per shape and options)
static void batch_mg_run(icarat_batch *B, int tile, int bpsm, double rtol, int maxit,
                         double refresh, int L, int warm)
{
  const auto key = std::make_tuple(tile, bpsm, rtol, maxit, refresh, L, warm);
  if(!B->mg_graph || B->mg_key != key)
  {
    if(B->mg_graph)
    {
      cudaGraphExecDestroy(B->mg_graph);
      B->mg_graph = nullptr;
    }
    cudaGraph_t g;
    ICK(cudaStreamBeginCapture(B->stream, cudaStreamCaptureModeThreadLocal));
    set_capturing(true);
    try
    {
      batch_mg_launch(B, tile, bpsm, rtol, maxit, refresh, L, warm);
    }
    catch(...)
    {
      set_capturing(false);
      cudaStreamEndCapture(B->stream, &g);
      throw;
    }
    set_capturing(false);
    ICK(cudaStreamEndCapture(B->stream, &g));
    ICK(cudaGraphInstantiate(&B->mg_graph, g, 0));
    cudaGraphDestroy(g);
    B->mg_key = key;
  }
  ICK(cudaGraphLaunch(B->mg_graph, B->stream));
  note_launch();
}

static int design_levels(const icarat_ctx *c, int want);

// Multigrid hierarchies of every design for the current designs (levels:
// the smallest count every design supports, at most `want`), the tables,
// and the batch stream ordered after the set-ups; cold starts clear x.
static int batch_mg_prepare(icarat_batch *B, int want, int tile, bool warm)
{
  IREQUIRE(want >= 2 && want <= kBmMaxLevels, ICARAT_ERR_ARG,
           "mg_levels must be in [2, 8] for the persistent multigrid launch");
  int L = want;
  for(icarat_ctx *c : B->ctx)
    L = std::min(L, design_levels(c, want));
  for(size_t d = 0; d < B->ctx.size(); d++)
  {
    icarat_ctx *c = B->ctx[d];
    c->mg_galerkin_req = 0; // the batch kernel runs the rediscretised hierarchy
    mg_setup(c, L, false);
    ICK(cudaEventRecord(B->ev[d], c->stream));
    ICK(cudaStreamWaitEvent(B->stream, B->ev[d], 0));
  }
  batch_mg_tables(B, L, tile);
  for(icarat_ctx *c : B->ctx)
    if(!warm || !c->have_u)
      ICK(cudaMemsetAsync(c->d_u, 0, sizeof(double) * c->neq, B->stream));
  return L;
}

static int pick_mg_tile(icarat_batch *B, const icarat_batch_opts *o)
{
  if(o && o->tile > 0)
    return o->tile;
  return B->mg_tuned_tile > 0 ? B->mg_tuned_tile : 256;
}

static int pick_mg_bpsm(icarat_batch *B, const icarat_batch_opts *o)
{
  if(o && o->blocks_per_sm > 0)
    return std::min(o->blocks_per_sm, B->occ_mg);
  return B->mg_tuned_bpsm > 0 ? B->mg_tuned_bpsm : B->occ_mg;
}

static int batch_collect(icarat_batch *B, double rtol, int maxit, icarat_solve_info *infos);

static int batch_solve_mg(icarat_batch *B, const icarat_batch_opts *o, double rtol, int maxit,
                          double refresh, icarat_solve_info *infos)
{
  const int tile = pick_mg_tile(B, o), bpsm = pick_mg_bpsm(B, o);
  IREQUIRE(tile >= 32 && tile <= (1 << 16), ICARAT_ERR_ARG, "tile must be in [32, 65536]");
  const bool warm = o && o->warm_start;
  const int L = batch_mg_prepare(B, o && o->mg_levels > 0 ? o->mg_levels : 4, tile, warm);
  batch_mg_run(B, tile, bpsm, rtol, maxit, refresh, L, warm ? 1 : 0);
  return batch_collect(B, rtol, maxit, infos);
}

static int batch_solve_impl(icarat_batch *B, const icarat_batch_opts *o,
                            icarat_solve_info *infos)
{
  const double rtol = o ? o->rtol : 1e-8;
  const int maxit = o && o->maxit > 0 ? o->maxit : 10000;
  const double refresh = o && o->refresh > 0.0 ? o->refresh : 1e-2;
  IREQUIRE(rtol >= 0.0 && refresh < 1.0, ICARAT_ERR_ARG, "bad batch options");
  const int method = o ? o->method : 0;
  IREQUIRE(method == 0 || method == ICARAT_SOLVER_MG_PCG || method == ICARAT_SOLVER_MIXED_IR,
           ICARAT_ERR_ARG, "batch method must be 0, ICARAT_SOLVER_MG_PCG or ICARAT_SOLVER_MIXED_IR");
  if(method == ICARAT_SOLVER_MIXED_IR)
    return batch_solve_concurrent(B, o, rtol, maxit, refresh, infos);
  if(method == ICARAT_SOLVER_MG_PCG)
    return batch_solve_mg(B, o, rtol, maxit, refresh, infos);
  const int tile = pick_tile(B, o), bpsm = pick_bpsm(B, o);
  IREQUIRE(tile >= 32 && tile <= (1 << 16), ICARAT_ERR_ARG, "tile must be in [32, 65536]");
  batch_run(B, tile, bpsm, rtol, maxit, refresh);
  return batch_collect(B, rtol, maxit, infos);
}

// per-design results of a persistent launch
static int batch_collect(icarat_batch *B, double rtol, int maxit, icarat_solve_info *infos)
{
  const size_t n = B->ctx.size();
  ICK(cudaMemcpyAsync(B->h_s, B->d_s, sizeof(BScal) * n, cudaMemcpyDeviceToHost, B->stream));
  ICK(cudaEventRecord(B->done_ev, B->stream));
  ICK(cudaStreamSynchronize(B->stream));
  int worst = ICARAT_OK;
  for(size_t d = 0; d < n; d++)
  {
    icarat_ctx *c = B->ctx[d];
    ICK(cudaStreamWaitEvent(c->stream, B->done_ev, 0));
    const BScal &S = B->h_s[d];
    icarat_solve_info si{};
    si.iterations = S.iter;
    si.rel_residual = S.bb > 0 ? std::sqrt(S.rr_true / S.bb) : 0.0;
    si.status = S.done ? S.status : ICARAT_WARN_MAXITER;
    si.refreshes = S.nrefresh;
    if(si.status == ICARAT_ERR_NAN || si.status == ICARAT_WARN_STAGNATION)
    {
      // the design's FP32 iteration stalled or broke down: FP64 MG-PCG
      // finishes it from the solution the launch left in the context (as
      // the single-design mixed solve does)
      icarat_solve_opts f{};
      f.method = ICARAT_SOLVER_MIXED_IR;
      f.rtol = rtol;
      f.maxit = maxit;
      f.mg_levels = B->mg_levels > 0 ? B->mg_levels : design_levels(c, 4);
      c->have_u = true;
      ICK(cudaStreamSynchronize(c->stream));
      mixed_fp64_finish(c, &f, c->d_rhs, c->d_u, &si, si.status);
    }
    note_result(c, si, infos ? &infos[d] : nullptr, worst);
  }
  return worst;
}

extern "C" {

int icarat_batch_create(const icarat_grid *grids, const icarat_bc *bcs, int count,
                        const icarat_material *mat, int device, icarat_batch **out)
{
  ICARAT_API_BEGIN
  IREQUIRE(grids && mat && out && count >= 1, ICARAT_ERR_ARG, "bad argument");
  *out = nullptr;
  icarat_batch *B = new icarat_batch;
  B->device = device;
  try
  {
    ICK(cudaSetDevice(device));
    ICK(cudaStreamCreateWithFlags(&B->stream, cudaStreamNonBlocking));
    const double h0[3] = {grids[0].lx / grids[0].nx, grids[0].ly / grids[0].ny,
                          grids[0].lz / grids[0].nz};
    for(int d = 0; d < count; d++)
    {
      const double h[3] = {grids[d].lx / grids[d].nx, grids[d].ly / grids[d].ny,
                           grids[d].lz / grids[d].nz};
      for(int q = 0; q < 3; q++)
        IREQUIRE(std::fabs(h[q] - h0[q]) <= 1e-12 * h0[q], ICARAT_ERR_UNSUPPORTED,
                 "batch members must share the element size");
      icarat_ctx *c = nullptr;
      const int st = icarat_ctx_create_impl(&grids[d], mat, bcs ? &bcs[d] : nullptr, device, &c);
      IREQUIRE(st == ICARAT_OK, st, "batch member creation failed");
      B->ctx.push_back(c);
      B->total_nv += 3L * c->numnp;
      cudaEvent_t e;
      ICK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
      B->ev.push_back(e);
    }
    ICK(cudaEventCreateWithFlags(&B->done_ev, cudaEventDisableTiming));
    B->ke = B->ctx[0]->ke0;
    B->kef = B->ctx[0]->ke0f;
    ICK(cudaMalloc(&B->buf, sizeof(float) * 6 * B->total_nv));
    ICK(cudaMalloc(&B->d_des, sizeof(BatchDesign) * count));
    ICK(cudaMalloc(&B->d_s, sizeof(BScal) * count));
    ICK(cudaMemset(B->d_s, 0, sizeof(BScal) * count));
    ICK(cudaMallocHost(&B->h_s, sizeof(BScal) * count));
    ICK(cudaMalloc(&B->d_ctl, sizeof(int) * 4));
    ICK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&B->occ, k_batch_pcg, kBatchThreads, 0));
    IREQUIRE(B->occ >= 1, ICARAT_ERR_CUDA, "batch kernel cannot be resident");
    ICK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&B->occ_mg, k_batch_mg, kBatchThreads,
                                                      0));
    IREQUIRE(B->occ_mg >= 1, ICARAT_ERR_CUDA, "batch multigrid kernel cannot be resident");
  }
  catch(...)
  {
    icarat_batch_destroy(B);
    throw;
  }
  *out = B;
  return ICARAT_OK;
  ICARAT_API_END
}

int icarat_batch_destroy(icarat_batch *B)
{
  if(!B)
    return ICARAT_OK;
  cudaSetDevice(B->device);
  if(B->stream)
    cudaStreamSynchronize(B->stream);
  if(B->graph)
    cudaGraphExecDestroy(B->graph);
  if(B->mg_graph)
    cudaGraphExecDestroy(B->mg_graph);
  for(int l = 1; l < kBmMaxLevels; l++)
    dfree(B->d_lv_items[l]);
  for(int l = 0; l < kBmMaxLevels; l++)
    dfree(B->d_lv_col[l]);
  dfree(B->d_partc);
  dfree(B->d_citems);
  dfree(B->d_y);
  dfree(B->d_bm);
  for(icarat_ctx *c : B->ctx)
    icarat_ctx_destroy(c);
  for(cudaEvent_t e : B->ev)
    cudaEventDestroy(e);
  if(B->done_ev)
    cudaEventDestroy(B->done_ev);
  for(void *p : {(void *)B->buf, (void *)B->d_des, (void *)B->d_item_design,
                 (void *)B->d_part, (void *)B->d_s, (void *)B->d_ctl})
    dfree(p);
  if(B->h_s)
    cudaFreeHost(B->h_s);
  if(B->stream)
    cudaStreamDestroy(B->stream);
  delete B;
  return ICARAT_OK;
}

int icarat_batch_ctx(icarat_batch *B, int i, icarat_ctx **ctx)
{
  ICARAT_API_BEGIN
  IREQUIRE(B && ctx && i >= 0 && i < (int)B->ctx.size(), ICARAT_ERR_ARG, "bad argument");
  *ctx = B->ctx[i];
  return ICARAT_OK;
  ICARAT_API_END
}

int icarat_batch_solve(icarat_batch *B, const icarat_batch_opts *opts,
                       icarat_solve_info *infos)
{
  ICARAT_API_BEGIN
  IREQUIRE(B, ICARAT_ERR_ARG, "null batch");
  ICK(cudaSetDevice(B->device));
  batch_prepare(B, true);
  return batch_solve_impl(B, opts, infos);
  ICARAT_API_END
}

int icarat_batch_solution(icarat_batch *B, int i, double *u)
{
  ICARAT_API_BEGIN
  IREQUIRE(B && u && i >= 0 && i < (int)B->ctx.size(), ICARAT_ERR_ARG, "bad argument");
  icarat_ctx *c = B->ctx[i];
  IREQUIRE(c->solved, ICARAT_ERR_STATE, "solve the batch first");
  from_full(c, c->d_u, u, true);
  return ICARAT_OK;
  ICARAT_API_END
}

int icarat_batch_autotune(icarat_batch *B, int *tile, int *bpsm, double *ms_per_iteration)
{
  ICARAT_API_BEGIN
  IREQUIRE(B, ICARAT_ERR_ARG, "null batch");
  ICK(cudaSetDevice(B->device));
  batch_prepare(B, true);
  // every candidate runs the same fixed work: 10 iterations of every design
  // (tolerance 0, cap 10) and the final FP64 refresh
  const int tiles[] = {128, 256, 512, 1024};
  double best = 1e30;
  int bt = 256, bb = B->occ;
  cudaEvent_t e0, e1;
  ICK(cudaEventCreate(&e0));
  ICK(cudaEventCreate(&e1));
  for(int tl : tiles)
    for(int bp = 1; bp <= B->occ; bp++)
    {
      batch_launch(B, tl, bp, 0.0, 10, 1e-2); // warm-up (and item tables)
      ICK(cudaEventRecord(e0, B->stream));
      batch_launch(B, tl, bp, 0.0, 10, 1e-2);
      ICK(cudaEventRecord(e1, B->stream));
      ICK(cudaEventSynchronize(e1));
      float ms = 0.f;
      ICK(cudaEventElapsedTime(&ms, e0, e1));
      if(ms < best)
      {
        best = ms;
        bt = tl;
        bb = bp;
      }
    }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  B->tile = bt;
  B->blocks_per_sm = bb;
  if(tile)
    *tile = bt;
  if(bpsm)
    *bpsm = bb;
  if(ms_per_iteration)
    *ms_per_iteration = best / 10.0;
  return ICARAT_OK;
  ICARAT_API_END
}

int icarat_batch_autotune_mg(icarat_batch *B, int mg_levels, int *tile, int *bpsm,
                             double *ms_per_iteration)
{
  ICARAT_API_BEGIN
  IREQUIRE(B, ICARAT_ERR_ARG, "null batch");
  ICK(cudaSetDevice(B->device));
  batch_prepare(B, true);
  // every candidate runs the same fixed work: 8 multigrid-PCG iterations of
  // every design (tolerance 0, cap 8) and the final FP64 refresh
  const int want = mg_levels > 0 ? mg_levels : 4;
  const int tiles[] = {128, 256, 512, 1024};
  double best = 1e30;
  int bt = 256, bb = B->occ_mg;
  cudaEvent_t e0, e1;
  ICK(cudaEventCreate(&e0));
  ICK(cudaEventCreate(&e1));
  for(int tl : tiles)
    for(int bp = 1; bp <= B->occ_mg; bp++)
    {
      const int L = batch_mg_prepare(B, want, tl, false);
      batch_mg_launch(B, tl, bp, 0.0, 8, 1e-2, L, 0); // warm-up
      ICK(cudaEventRecord(e0, B->stream));
      batch_mg_launch(B, tl, bp, 0.0, 8, 1e-2, L, 0);
      ICK(cudaEventRecord(e1, B->stream));
      ICK(cudaEventSynchronize(e1));
      float ms = 0.f;
      ICK(cudaEventElapsedTime(&ms, e0, e1));
      if(ms < best)
      {
        best = ms;
        bt = tl;
        bb = bp;
      }
    }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  B->mg_tuned_tile = bt;
  B->mg_tuned_bpsm = bb;
  if(tile)
    *tile = bt;
  if(bpsm)
    *bpsm = bb;
  if(ms_per_iteration)
    *ms_per_iteration = best / 8.0;
  return ICARAT_OK;
  ICARAT_API_END
}

int icarat_batch_loop_step(icarat_batch *B, const icarat_batch_opts *opts,
                           icarat_step_info *infos)
{
  ICARAT_API_BEGIN
  IREQUIRE(B, ICARAT_ERR_ARG, "null batch");
  ICK(cudaSetDevice(B->device));
  const size_t n = B->ctx.size();
  for(size_t d = 0; d < n; d++)
    IREQUIRE(B->ctx[d]->loop.ncases == 0, ICARAT_ERR_UNSUPPORTED,
             "batch members take one load case each (icarat_loop_step runs several)");
  std::vector<double> beta(n);
  for(size_t d = 0; d < n; d++)
    beta[d] = loop_pre(B->ctx[d]); // filter, design, right-hand side
  batch_prepare(B, false);
  std::vector<icarat_solve_info> si(n);
  batch_solve_impl(B, opts, si.data());
  int worst = ICARAT_OK;
  for(size_t d = 0; d < n; d++)
  {
    const int st = loop_post(B->ctx[d], si[d].status, si[d], beta[d], infos ? &infos[d] : nullptr);
    if(st < 0)
      worst = std::min(worst, st);
    else if(worst >= 0 && st > worst)
      worst = st;
  }
  return worst;
  ICARAT_API_END
}

} // extern "C"
