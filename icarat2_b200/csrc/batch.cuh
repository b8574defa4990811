// Shared pieces of the batched persistent solvers (batch.cu: Jacobi-PCG,
// batch_mg.cu: multigrid-PCG): the design table, the per-design scalars, the
// launch arguments and the device helpers both kernels use.
#pragma once
#include <cooperative_groups.h>

#include "stencil.cuh"

namespace icarat_b200
{

struct BatchDesign
{
  GridDev g;
  const float *E32;
  const double *E64;
  const uint8_t *fix;
  const double *b;
  double *x64;
  long off;   // first entry of this design in the FP32 node buffers
  int item0;  // first work item
  int nitems; // work items
};

struct BScal
{
  double rz, bb, rr_ref, rr_true, tol2, delta2;
  double rr_nat; // FP64 r . r at the last refresh the design asked for itself
  int iter, maxit, done, status, refresh, final_, nrefresh, nstall;
  int last_refresh; // iteration of the last FP64 residual
};

struct BatchArgs
{
  KeParam ke;
  KeParamF kef;
  const BatchDesign *des;
  int ndes;
  const int *item_design;
  int nitems, tile;
  float *x32, *r, *z, *p, *Ap, *invd;
  double *part; // 4 per item
  BScal *s;
  int *ctl; // [0] designs still iterating, [1], [2] refresh requests by parity
  int maxit;
  double tol, delta;
};

constexpr int kBatchThreads = 128;

// Sum of partial k over the items of design D, in item order; every thread
// of the block gets the result.
__device__ __forceinline__ double design_sum(const BatchArgs &a, const BatchDesign &D, int k, double *sh,
                             double *bc)
{
  double v = 0.0;
  for(int i = threadIdx.x; i < D.nitems; i += blockDim.x)
    v += __ldcg(a.part + 4L * (D.item0 + i) + k);
  double arr[1] = {v};
  block_sum<1>(arr, sh);
  if(threadIdx.x == 0)
    *bc = arr[0];
  __syncthreads();
  const double r = *bc;
  __syncthreads();
  return r;
}

// (K x)_n in FP64 element by element: few live registers, for the refresh
// phase, which runs rarely and must not raise the register count of the
// whole persistent kernel.  Coherent (L2) loads: x changes inside the launch.
__device__ __forceinline__ void node_Ku_lean(const GridDev &g, const KeParam &ke,
                                             const double *__restrict__ E,
                                             const double *__restrict__ x, int n,
                                             double (&acc)[3])
{
  const int i = n % g.NX, j = (n / g.NX) % g.NY, k = n / (g.NX * g.NY);
  acc[0] = acc[1] = acc[2] = 0.0;
#pragma unroll
  for(int sz = 0; sz < 2; sz++)
#pragma unroll
    for(int sy = 0; sy < 2; sy++)
#pragma unroll
      for(int sx = 0; sx < 2; sx++)
      {
        const int ei = i - 1 + sx, ej = j - 1 + sy, ek = k - 1 + sz;
        const double e = load_E(E, g, ei, ej, ek);
        if(e == 0.0)
          continue;
        const int la = local_node(1 - sx, 1 - sy, 1 - sz);
        double t[3] = {0.0, 0.0, 0.0};
#pragma unroll
        for(int bz = 0; bz < 2; bz++)
#pragma unroll
          for(int by = 0; by < 2; by++)
#pragma unroll
            for(int bx = 0; bx < 2; bx++)
            {
              const int lb = local_node(bx, by, bz);
              const long m = (long)(ei + bx) + (long)(ej + by) * g.NX +
                             (long)(ek + bz) * g.NX * g.NY;
#pragma unroll
              for(int d = 0; d < 3; d++)
              {
                const double u = __ldcg(x + (long)d * g.numnp + m);
#pragma unroll
                for(int c = 0; c < 3; c++)
                  t[c] = fma(ke.k[(3 * la + c) * 24 + 3 * lb + d], u, t[c]);
              }
            }
#pragma unroll
        for(int c = 0; c < 3; c++)
          acc[c] = fma(e, t[c], acc[c]);
      }
}


constexpr int kBmMaxLevels = 8;
constexpr int kBmMaxDeg = 4;

// one multigrid level of one design (FP32 operator and work vectors)
struct BmLevel
{
  GridDev g;
  const float *E32, *invd;
  const uint8_t *fix;
  float *x, *t, *r, *b; // iterate, its alternate, residual / Chebyshev d, right-hand side
  int item0, nitems;     // node tiles of this level in the level's item table
  // column items of the stencil phases: blocks of kBatchThreads node
  // columns (i, j) times chunks of kc node layers, in the level's column table
  int mitem0, mitems, ncb, kc;
};

// the multigrid hierarchy of one design: levels, the coarsest level's dense
// solve x = W^T (W b) (W = L^-1 of the coarse Cholesky factor, FP64, row
// major, and its transpose), and the Chebyshev coefficients of its smoother
struct BmDesign
{
  BmLevel lv[kBmMaxLevels];
  const double *W, *WT;
  const int *map;  // coarse unknown -> index of the coarsest level's node vectors
  const int *cmap; // node-major index 3 n + q of the coarsest level -> unknown (-1: fixed)
  double *v;       // the coarsest right-hand side gathered to the unknowns
  double *y;       // W v
  int nc;         // coarse unknowns
  int citem0, citems;
  float inv_theta;
  float pre_c1[kBmMaxDeg], pre_c2[kBmMaxDeg], post_c1[kBmMaxDeg], post_c2[kBmMaxDeg];
};

struct BmArgs
{
  int levels, deg, ctile;
  int warm; // start from each design's x64 (r = b - K x in FP64) instead of 0
  const BmDesign *bm;
  const int *lv_item_design[kBmMaxLevels]; // per level: item -> design
  int lv_nitems[kBmMaxLevels];
  const int *c_item_design; // coarse row items -> design
  int c_nitems;
  const int *lv_col_design[kBmMaxLevels]; // per level: column item -> design
  int lv_col_items[kBmMaxLevels];
  double *partc; // 4 per finest-level column item: p.Ap, z.r, z.Ap
};

// sum of partial k over items [i0, i0 + n) of `part` (4 per item), in item
// order; every thread of the block gets the result
__device__ __forceinline__ double range_sum(const double *part, int i0, int n, int k,
                                            double *sh, double *bc)
{
  double v = 0.0;
  for(int i = threadIdx.x; i < n; i += blockDim.x)
    v += __ldcg(part + 4L * (i0 + i) + k);
  double arr[1] = {v};
  block_sum<1>(arr, sh);
  if(threadIdx.x == 0)
    *bc = arr[0];
  __syncthreads();
  const double r = *bc;
  __syncthreads();
  return r;
}

__global__ void k_batch_mg(BatchArgs a, BmArgs m);

} // namespace icarat_b200
