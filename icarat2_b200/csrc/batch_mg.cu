// Batched multigrid-preconditioned CG of many independent designs in ONE
// persistent cooperative launch (no reference counterpart; the reference
// solves one design at a time with Jacobi-PCG, solvers.cpp:63-91).
//
// Every design keeps the geometric multigrid hierarchy its context builds
// (mg_setup: rediscretised SIMP moduli, Jacobi diagonals, the coarsest
// level's dense inverse factor W = L^-1).  The launch iterates all designs
// together over work items: node tiles of every level of every design, and
// row blocks of every design's coarsest dense solve.  Each phase below walks
// its item table (a contiguous run per CTA) and ends at a grid-wide barrier,
// so designs of different sizes share the GPU in proportion to their work:
//
//   P1  Ap = K p (FP32 column-march stencil), partial p . Ap
//   P2  alpha; x32 += alpha p, r -= alpha Ap, partial r . r; and the first
//       Chebyshev step of the finest level from zero, x = d = D^-1 r / theta
//   F   the FP64 refresh decision of each design (r . r fell by the factor
//       `refresh` below the last FP64 residual, below the target, or the
//       iteration cap); x += x32, x32 = 0 for the designs that refresh
//   R   (only when some design refreshes) r = b - K x in FP64 for those
//       designs, and their first Chebyshev step redone from that r
//   V   z = M r: one V-cycle over all designs (per level down: deg-1
//       Chebyshev steps, residual, restriction fused with the next level's
//       first Chebyshev step; coarsest: y = W b, x = W^T y; per level up:
//       prolongation, deg Chebyshev steps; the finest level's last step
//       writes z with the partials z . r and z . Ap)
//   P3  beta = -z.Ap / p.Ap (flexible CG), p = z + beta p; after a refresh
//       the design's first item takes the stop test on the FP64 residual
// The refresh replaces the FP32 recurrence residual by the FP64 one before
// the V-cycle, as the single-design mixed-precision solver does: the search
// direction survives it and no extra V-cycle is spent.  Vectors and the
// V-cycle are FP32 (as the mixed-precision solver's); the solution,
// right-hand side, dot products and scalars are FP64; the coarse dense solve
// is FP64.  Every grid barrier is reached by every CTA the same number of
// times; the loop is capped at maxit + 2 iterations.
#include "batch.cuh"

namespace cg = cooperative_groups;

namespace icarat_b200
{

namespace
{
struct Span
{
  int i0, i1;
};

__device__ __forceinline__ Span span_of(int nitems)
{
  const int ipb = (nitems + gridDim.x - 1) / gridDim.x;
  Span s;
  s.i0 = min((int)blockIdx.x * ipb, nitems);
  s.i1 = min(s.i0 + ipb, nitems);
  return s;
}

// design d takes part in a phase: not done, and (refresh mode) refreshing
__device__ __forceinline__ bool takes_part(const BatchArgs &a, int d, int mode)
{
  const BScal &S = a.s[d];
  if(*(volatile const int *)&S.done)
    return false;
  return mode == 0 || *(volatile const int *)&S.refresh;
}
// takes_part, read by thread 0 and shared with the block: for a phase in
// which another CTA may set the design's done flag (P3), so that every
// thread of the block takes the same branch around the block reductions
__device__ __forceinline__ bool takes_part_block(const BatchArgs &a, int d, int mode, int *flag)
{
  if(threadIdx.x == 0)
    *flag = takes_part(a, d, mode) ? 1 : 0;
  __syncthreads();
  const bool r = *flag != 0;
  __syncthreads();
  return r;
}

// node column and z range of this thread in column item q of a level (q
// counted from the level's first column item; ncb column blocks, chunks of
// kc node layers); false for the columns past the level's last
__device__ __forceinline__ bool col_item(const GridDev &g, int q, int ncb, int kc, int &i, int &j,
                                         int &k0, int &k1)
{
  const int col = (q % ncb) * kBatchThreads + (int)threadIdx.x;
  k0 = (q / ncb) * kc;
  k1 = min(k0 + kc, g.NZ);
  if(col >= g.NX * g.NY)
    return false;
  i = col % g.NX;
  j = col / g.NX;
  return true;
}

// the finest level's first Chebyshev step from zero, x = d = D^-1 r / theta,
// with the design's fields held in registers across a phase's nodes
struct Step0
{
  float inv_theta;
  const float *invd;
  float *x, *d;
  __device__ __forceinline__ void operator()(long id, float ri) const
  {
    const float di = inv_theta * __ldg(invd + id) * ri;
    x[id] = di;
    d[id] = di;
  }
};

__device__ __forceinline__ Step0 step0_of(const BmDesign &B)
{
  return Step0{B.inv_theta, B.lv[0].invd, B.lv[0].x, B.lv[0].r};
}

// nodes a thread has in flight in the elementwise phases: all loads of kU
// nodes are issued before the first store, so a thread waits for memory
// once per kU nodes rather than once per component
constexpr int kU = 4;

// y = c x + y (c = 0: y = x) over the nodes [n0, n1) of one design's three
// component blocks (stride numnp)
__device__ __forceinline__ void xpby_nodes(float *y, const float *x, float c, int numnp, int n0,
                                           int n1)
{
  for(int nb = n0 + (int)threadIdx.x; nb < n1; nb += kU * (int)blockDim.x)
  {
    float xv[kU][3], yv[kU][3];
#pragma unroll
    for(int u = 0; u < kU; u++)
    {
      const int n = nb + u * (int)blockDim.x;
#pragma unroll
      for(int q = 0; q < 3; q++)
      {
        const long id = (long)q * numnp + n;
        xv[u][q] = n < n1 ? __ldcg(x + id) : 0.0f;
        yv[u][q] = (n < n1 && c != 0.0f) ? __ldcg(y + id) : 0.0f;
      }
    }
#pragma unroll
    for(int u = 0; u < kU; u++)
    {
      const int n = nb + u * (int)blockDim.x;
      if(n < n1)
#pragma unroll
        for(int q = 0; q < 3; q++)
          y[(long)q * numnp + n] = fmaf(c, yv[u][q], xv[u][q]);
    }
  }
}
} // namespace

__global__ void __launch_bounds__(kBatchThreads, 4) k_batch_mg(BatchArgs a, BmArgs m)
{
  cg::grid_group grid = cg::this_grid();
  __shared__ double sh[4 * 32];
  __shared__ double bc[4];
  __shared__ int part_flag;
  const int t = threadIdx.x;
  const int L = m.levels;
  const Span s0 = span_of(a.nitems);
  // iterate of each level: 0 in x, 1 in t (the same in every thread)
  int cur[kBmMaxLevels];
  for(int l = 0; l < kBmMaxLevels; l++)
    cur[l] = 0;

  if(blockIdx.x == 0 && t == 0)
  {
    a.ctl[0] = a.ndes;
    a.ctl[1] = a.ctl[2] = 0;
  }

  // one Chebyshev step on level l of the designs in `mode`:
  // d = c1 d + c2 D^-1 (b - K x), xo = x + d; on the finest level's last
  // step (fin) xo is z and the partials z . r (slot 1) and z . Ap (slot 2)
  // are written
  auto cheb = [&](int l, int mode, bool post, int k, bool fin)
  {
    const Span sp = span_of(m.lv_col_items[l]);
    const int c = cur[l];
    // the design's fields in registers, reloaded when the item's design
    // changes: the stores below would otherwise make every use reload them
    int cd = -1, mitem0 = 0, ncb = 0, kc = 0;
    bool part = false;
    GridDev g{};
    float c1 = 0.0f, c2 = 0.0f;
    const float *x = nullptr, *b = nullptr, *ap = nullptr, *invd = nullptr, *E = nullptr;
    float *xo = nullptr, *dv = nullptr;
    const uint8_t *fix = nullptr;
    for(int item = sp.i0; item < sp.i1; item++)
    {
      const int d = m.lv_col_design[l][item];
      if(d != cd)
      {
        cd = d;
        part = takes_part(a, d, mode);
        const BmDesign &B = m.bm[d];
        const BmLevel &Lv = B.lv[l];
        const long off = a.des[d].off;
        g = Lv.g;
        c1 = post ? B.post_c1[k] : B.pre_c1[k];
        c2 = post ? B.post_c2[k] : B.pre_c2[k];
        x = c ? Lv.t : Lv.x;
        xo = fin ? a.z + off : (c ? Lv.x : Lv.t);
        b = l == 0 ? a.r + off : Lv.b;
        ap = a.Ap + off;
        dv = Lv.r;
        invd = Lv.invd;
        fix = Lv.fix;
        E = Lv.E32;
        mitem0 = Lv.mitem0;
        ncb = Lv.ncb;
        kc = Lv.kc;
      }
      if(!part)
        continue;
      double rz = 0.0, zap = 0.0;
      int i, j, k0, k1;
      if(col_item(g, item - mitem0, ncb, kc, i, j, k0, k1))
      {
        const int n_ij = i + j * g.NX, nxy = g.NX * g.NY;
        column_Ku<float, KeParamF, true>(
            g, a.kef, E, x, i, j, k0, k1,
            [&](int kk, const float(&acc)[3], const float(&uc)[3])
            {
              const int n = n_ij + kk * nxy;
              const unsigned f = fix[n];
#pragma unroll
              for(int q = 0; q < 3; q++)
              {
                const long id = (long)q * g.numnp + n;
                float dn = 0.0f;
                if(!((f >> q) & 1u))
                  dn = (c1 != 0.0f ? c1 * __ldcg(dv + id) : 0.0f) +
                       c2 * __ldg(invd + id) * (__ldcg(b + id) - acc[q]);
                dv[id] = dn;
                const float xn = uc[q] + dn;
                xo[id] = xn;
                if(fin)
                {
                  rz += (double)xn * (double)__ldcg(b + id);
                  zap += (double)xn * (double)__ldcg(ap + id);
                }
              }
            });
      }
      if(fin)
      {
        double v[2] = {rz, zap};
        block_sum<2>(v, sh);
        if(t == 0)
        {
          m.partc[4L * item + 1] = v[0];
          m.partc[4L * item + 2] = v[1];
        }
        __syncthreads();
      }
    }
    cur[l] ^= 1;
  };

  // r_l = b_l - K x_l
  auto residual = [&](int l, int mode)
  {
    const Span sp = span_of(m.lv_col_items[l]);
    const int c = cur[l];
    int cd = -1, mitem0 = 0, ncb = 0, kc = 0;
    bool part = false;
    GridDev g{};
    const float *x = nullptr, *b = nullptr, *E = nullptr;
    float *r = nullptr;
    const uint8_t *fix = nullptr;
    for(int item = sp.i0; item < sp.i1; item++)
    {
      const int d = m.lv_col_design[l][item];
      if(d != cd)
      {
        cd = d;
        part = takes_part(a, d, mode);
        const BmLevel &Lv = m.bm[d].lv[l];
        g = Lv.g;
        x = c ? Lv.t : Lv.x;
        b = l == 0 ? a.r + a.des[d].off : Lv.b;
        r = Lv.r;
        fix = Lv.fix;
        E = Lv.E32;
        mitem0 = Lv.mitem0;
        ncb = Lv.ncb;
        kc = Lv.kc;
      }
      if(!part)
        continue;
      int i, j, k0, k1;
      if(col_item(g, item - mitem0, ncb, kc, i, j, k0, k1))
      {
        const int n_ij = i + j * g.NX, nxy = g.NX * g.NY;
        column_Ku<float, KeParamF, true>(
            g, a.kef, E, x, i, j, k0, k1,
            [&](int kk, const float(&acc)[3], const float(&)[3])
            {
              const int n = n_ij + kk * nxy;
              const unsigned f = fix[n];
#pragma unroll
              for(int q = 0; q < 3; q++)
              {
                const long id = (long)q * g.numnp + n;
                r[id] = ((f >> q) & 1u) ? 0.0f : __ldcg(b + id) - acc[q];
              }
            });
      }
    }
  };

  // b_{l+1} = R r_l, and (above the coarsest level) the first Chebyshev
  // step of level l + 1 from zero
  auto restrict_to = [&](int l, int mode)
  {
    const int lc = l + 1;
    const bool smooth = lc < L - 1;
    const Span sp = span_of(m.lv_nitems[lc]);
    for(int item = sp.i0; item < sp.i1; item++)
    {
      const int d = m.lv_item_design[lc][item];
      if(!takes_part(a, d, mode))
        continue;
      const BmDesign &B = m.bm[d];
      const BmLevel &F = B.lv[l], &C = B.lv[lc];
      const GridDev gf = F.g, gc = C.g;
      const float *rf = F.r;
      const uint8_t *fix = C.fix;
      float *bc_ = C.b;
      const int *cmap = B.cmap;
      double *v = B.v;
      const float inv_theta = B.inv_theta;
      const float *invd = C.invd;
      float *xc = C.x, *dc = C.r;
      const int n0 = (item - C.item0) * a.tile, n1 = min(n0 + a.tile, gc.numnp);
      for(int n = n0 + t; n < n1; n += blockDim.x)
      {
        float sr[3];
        restrict_node<float, true>(gf, gc, rf, n, sr);
        const unsigned fx = fix[n];
#pragma unroll
        for(int q = 0; q < 3; q++)
        {
          const long id = (long)q * gc.numnp + n;
          const float bq = ((fx >> q) & 1u) ? 0.0f : sr[q];
          bc_[id] = bq;
          if(!smooth)
          {
            // coarsest level: the dense solve's right-hand side, gathered
            const int u = __ldg(cmap + 3L * n + q);
            if(u >= 0)
              v[u] = (double)bq;
          }
          else
          {
            const float di = inv_theta * __ldg(invd + id) * bq;
            xc[id] = di;
            dc[id] = di;
          }
        }
      }
    }
    cur[lc] = 0;
  };

  // coarsest level: y = W v (and the level's iterate cleared), then x = W^T y
  auto coarse_lower = [&](int mode)
  {
    const Span sp = span_of(m.c_nitems);
    const int warp = t >> 5, lane = t & 31, nw = blockDim.x >> 5;
    for(int item = sp.i0; item < sp.i1; item++)
    {
      const int d = m.c_item_design[item];
      if(!takes_part(a, d, mode))
        continue;
      const BmDesign &B = m.bm[d];
      const int nc = B.nc, citems = B.citems;
      const double *W = B.W, *v = B.v;
      double *y = B.y;
      float *xc = B.lv[L - 1].x;
      const long nv = 3L * B.lv[L - 1].g.numnp;
      const int q = item - B.citem0;
      const int r0 = q * m.ctile, r1 = min(r0 + m.ctile, nc);
      // rows ra and rb = ra + nw of the item together: eight loads of W and
      // of v in flight per lane (four independent partial sums per row)
      for(int ra = r0 + warp; ra < r1; ra += 2 * nw)
      {
        const int rb = ra + nw < r1 ? ra + nw : -1;
        const double *rowa = W + (long)ra * nc, *rowb = W + (long)(rb < 0 ? ra : rb) * nc;
        const int lenb = rb < 0 ? 0 : rb + 1;
        double sa[4] = {0.0, 0.0, 0.0, 0.0}, sb[4] = {0.0, 0.0, 0.0, 0.0};
        int j = lane;
        for(; j + 96 <= ra; j += 128)
#pragma unroll
          for(int u = 0; u < 4; u++)
          {
            const double vj = __ldcg(v + j + 32 * u);
            sa[u] = fma(__ldg(rowa + j + 32 * u), vj, sa[u]);
            sb[u] = fma(__ldg(rowb + j + 32 * u), vj, sb[u]);
          }
        // the rest of row ra (its last entry is column ra)
        for(int jj = j; jj <= ra; jj += 32)
          sa[0] = fma(__ldg(rowa + jj), __ldcg(v + jj), sa[0]);
        // the rest of row rb (rb > ra: longer)
        for(; j + 96 < lenb; j += 128)
#pragma unroll
          for(int u = 0; u < 4; u++)
            sb[u] = fma(__ldg(rowb + j + 32 * u), __ldcg(v + j + 32 * u), sb[u]);
        for(; j < lenb; j += 32)
          sb[0] = fma(__ldg(rowb + j), __ldcg(v + j), sb[0]);
        double suma = (sa[0] + sa[1]) + (sa[2] + sa[3]);
        double sumb = (sb[0] + sb[1]) + (sb[2] + sb[3]);
        for(int o = 16; o > 0; o >>= 1)
        {
          suma += __shfl_xor_sync(0xffffffffu, suma, o);
          sumb += __shfl_xor_sync(0xffffffffu, sumb, o);
        }
        if(lane == 0)
        {
          y[ra] = suma;
          if(rb >= 0)
            y[rb] = sumb;
        }
      }
      // this item's share of the coarsest iterate, cleared (constrained
      // entries stay 0; the free ones are written below)
      const long per = (nv + citems - 1) / citems;
      const long e0 = (long)q * per, e1 = min(e0 + per, nv);
      for(long e = e0 + t; e < e1; e += blockDim.x)
        xc[e] = 0.0f;
    }
    cur[L - 1] = 0;
  };
  auto coarse_upper = [&](int mode)
  {
    const Span sp = span_of(m.c_nitems);
    const int warp = t >> 5, lane = t & 31, nw = blockDim.x >> 5;
    for(int item = sp.i0; item < sp.i1; item++)
    {
      const int d = m.c_item_design[item];
      if(!takes_part(a, d, mode))
        continue;
      const BmDesign &B = m.bm[d];
      const int nc = B.nc;
      const double *WT = B.WT, *y = B.y;
      const int *map = B.map;
      float *xc = B.lv[L - 1].x;
      const int q = item - B.citem0;
      const int r0 = q * m.ctile, r1 = min(r0 + m.ctile, nc);
      // rows ra and rb = ra + nw together, as in the lower solve (row r of
      // W^T holds columns r .. nc - 1)
      for(int ra = r0 + warp; ra < r1; ra += 2 * nw)
      {
        const int rb = ra + nw < r1 ? ra + nw : nc; // nc: no second row
        const double *rowa = WT + (long)ra * nc, *rowb = WT + (long)(rb < nc ? rb : ra) * nc;
        double sa[4] = {0.0, 0.0, 0.0, 0.0}, sb[4] = {0.0, 0.0, 0.0, 0.0};
        int ja = ra + lane, jb = rb + lane;
        for(; jb + 96 < nc; ja += 128, jb += 128)
#pragma unroll
          for(int u = 0; u < 4; u++)
          {
            sa[u] = fma(__ldg(rowa + ja + 32 * u), __ldcg(y + ja + 32 * u), sa[u]);
            sb[u] = fma(__ldg(rowb + jb + 32 * u), __ldcg(y + jb + 32 * u), sb[u]);
          }
        for(; ja + 96 < nc; ja += 128)
#pragma unroll
          for(int u = 0; u < 4; u++)
            sa[u] = fma(__ldg(rowa + ja + 32 * u), __ldcg(y + ja + 32 * u), sa[u]);
        for(; ja < nc; ja += 32)
          sa[0] = fma(__ldg(rowa + ja), __ldcg(y + ja), sa[0]);
        for(; jb < nc; jb += 32)
          sb[0] = fma(__ldg(rowb + jb), __ldcg(y + jb), sb[0]);
        double suma = (sa[0] + sa[1]) + (sa[2] + sa[3]);
        double sumb = (sb[0] + sb[1]) + (sb[2] + sb[3]);
        for(int o = 16; o > 0; o >>= 1)
        {
          suma += __shfl_xor_sync(0xffffffffu, suma, o);
          sumb += __shfl_xor_sync(0xffffffffu, sumb, o);
        }
        if(lane == 0)
        {
          xc[__ldg(map + ra)] = (float)suma;
          if(rb < nc)
            xc[__ldg(map + rb)] = (float)sumb;
        }
      }
    }
  };

  // x_l += P x_{l+1}
  auto prolong = [&](int l, int mode)
  {
    const Span sp = span_of(m.lv_nitems[l]);
    const int c = cur[l], cc = cur[l + 1];
    for(int item = sp.i0; item < sp.i1; item++)
    {
      const int d = m.lv_item_design[l][item];
      if(!takes_part(a, d, mode))
        continue;
      const BmDesign &B = m.bm[d];
      const BmLevel &F = B.lv[l], &C = B.lv[l + 1];
      const GridDev gf = F.g, gc = C.g;
      float *x = c ? F.t : F.x;
      const float *xc = cc ? C.t : C.x;
      const uint8_t *fix = F.fix;
      const int n0 = (item - F.item0) * a.tile, n1 = min(n0 + a.tile, gf.numnp);
      for(int n = n0 + t; n < n1; n += blockDim.x)
      {
        float s[3];
        prolong_node<float, true>(gf, gc, xc, n, s);
        const unsigned fx = fix[n];
#pragma unroll
        for(int q = 0; q < 3; q++)
          if(!((fx >> q) & 1u))
          {
            const long id = (long)q * gf.numnp + n;
            x[id] = __ldcg(x + id) + s[q];
          }
      }
    }
  };

  // z = M r for the designs in `mode` (the finest level's first step from
  // zero was fused into the phase that wrote r)
  auto vcycle = [&](int mode)
  {
    cur[0] = 0;
    for(int l = 0; l < L - 1; l++)
    {
      for(int k = 1; k < m.deg; k++)
      {
        cheb(l, mode, false, k, false);
        grid.sync();
      }
      residual(l, mode);
      grid.sync();
      restrict_to(l, mode);
      grid.sync();
    }
    coarse_lower(mode);
    grid.sync();
    coarse_upper(mode);
    grid.sync();
    for(int l = L - 2; l >= 0; l--)
    {
      prolong(l, mode);
      grid.sync();
      for(int k = 0; k < m.deg; k++)
      {
        cheb(l, mode, true, k, l == 0 && k == m.deg - 1);
        grid.sync();
      }
    }
  };

  // ---- init: x = 0 (or the design's x, warm), x32 = 0, r = b - K x, first
  // smoothing step; partial b . b
  for(int item = s0.i0; item < s0.i1; item++)
  {
    const int d = a.item_design[item];
    const BatchDesign &D = a.des[d];
    const BmDesign &B = m.bm[d];
    const int n0 = (item - D.item0) * a.tile;
    double bb = 0.0;
    // the FP64 node stencil leaves no registers to hold the design's fields:
    // they are read from the tables (this phase runs once per solve)
    for(int n = n0 + t; n < min(n0 + a.tile, D.g.numnp); n += blockDim.x)
    {
      const unsigned f = D.fix[n];
      double acc[3] = {0.0, 0.0, 0.0};
      if(m.warm)
        node_Ku_lean(D.g, a.ke, D.E64, D.x64, n, acc);
#pragma unroll
      for(int c = 0; c < 3; c++)
      {
        const long id = (long)c * D.g.numnp + n, o = D.off + id;
        const double bi = ((f >> c) & 1u) ? 0.0 : D.b[id];
        const float ri = ((f >> c) & 1u) ? 0.0f : (float)(bi - acc[c]);
        a.x32[o] = 0.0f;
        a.r[o] = ri;
        step0_of(B)(id, ri);
        bb += bi * bi;
      }
    }
    double v[1] = {bb};
    block_sum<1>(v, sh);
    if(t == 0)
      a.part[4L * item + 3] = v[0];
    __syncthreads();
  }
  grid.sync();
  for(int item = s0.i0; item < s0.i1; item++)
  {
    const int d = a.item_design[item];
    const BatchDesign &D = a.des[d];
    if(item != D.item0)
      continue;
    const double bb = design_sum(a, D, 3, sh, bc);
    if(t == 0)
    {
      BScal &S = a.s[d];
      S.bb = bb;
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
  // ---- z = M r, p = z, z . r
  vcycle(0);
  {
    int cd = -1, numnp = 0, item0 = 0;
    long off = 0;
    bool part = false;
    for(int item = s0.i0; item < s0.i1; item++)
    {
      const int d = a.item_design[item];
      if(d != cd)
      {
        cd = d;
        part = takes_part(a, d, 0);
        const BatchDesign &D = a.des[d];
        numnp = D.g.numnp;
        off = D.off;
        item0 = D.item0;
      }
      if(!part)
        continue;
      if(item == item0)
      {
        const BmLevel &L0 = m.bm[d].lv[0];
        const double rz = range_sum(m.partc, L0.mitem0, L0.mitems, 1, sh, bc);
        if(t == 0)
          a.s[d].rz = rz;
      }
      const int n0 = (item - item0) * a.tile, n1 = min(n0 + a.tile, numnp);
      xpby_nodes(a.p + off, a.z + off, 0.0f, numnp, n0, n1);
    }
  }
  grid.sync();

  for(int it = 0; it < a.maxit + 2; it++)
  {
    if(*(volatile int *)&a.ctl[0] <= 0)
      break;
    // ---- P1: Ap = K p, partial p . Ap (finest-level column items)
    {
      const Span sp = span_of(m.lv_col_items[0]);
      int cd = -1, mitem0 = 0, ncb = 0, kc = 0;
      bool part = false;
      GridDev g{};
      const float *E = nullptr, *p = nullptr;
      float *ap = nullptr;
      const uint8_t *fix = nullptr;
      for(int item = sp.i0; item < sp.i1; item++)
      {
        const int d = m.lv_col_design[0][item];
        if(d != cd)
        {
          cd = d;
          part = takes_part(a, d, 0);
          const BatchDesign &D = a.des[d];
          const BmLevel &Lv = m.bm[d].lv[0];
          g = D.g;
          E = D.E32;
          p = a.p + D.off;
          ap = a.Ap + D.off;
          fix = D.fix;
          mitem0 = Lv.mitem0;
          ncb = Lv.ncb;
          kc = Lv.kc;
        }
        if(!part)
          continue;
        double pap = 0.0;
        int i, j, k0, k1;
        if(col_item(g, item - mitem0, ncb, kc, i, j, k0, k1))
        {
          const int n_ij = i + j * g.NX, nxy = g.NX * g.NY;
          column_Ku<float, KeParamF, true>(
              g, a.kef, E, p, i, j, k0, k1,
              [&](int kk, const float(&acc)[3], const float(&uc)[3])
              {
                const int n = n_ij + kk * nxy;
                const unsigned f = fix[n];
#pragma unroll
                for(int c = 0; c < 3; c++)
                {
                  const float y = ((f >> c) & 1u) ? 0.0f : acc[c];
                  ap[(long)c * g.numnp + n] = y;
                  pap += (double)uc[c] * (double)y;
                }
              });
        }
        double v[1] = {pap};
        block_sum<1>(v, sh);
        if(t == 0)
          m.partc[4L * item] = v[0];
        __syncthreads();
      }
    }
    grid.sync();
    // ---- P2: alpha; x32 += alpha p, r -= alpha Ap, partial r . r (slot 3);
    // the first smoothing step of the V-cycle below
    {
      int cd = -1, numnp = 0, item0 = 0;
      long off = 0;
      bool part = false;
      float al = 0.0f;
      Step0 st{};
      for(int item = s0.i0; item < s0.i1; item++)
      {
        const int d = a.item_design[item];
        if(d != cd)
        {
          cd = d;
          part = takes_part(a, d, 0);
          if(part)
          {
            const BatchDesign &D = a.des[d];
            const BmDesign &B = m.bm[d];
            const double pap =
                range_sum(m.partc, B.lv[0].mitem0, B.lv[0].mitems, 0, sh, bc);
            al = (float)(a.s[d].rz / pap);
            numnp = D.g.numnp;
            off = D.off;
            item0 = D.item0;
            st = step0_of(B);
          }
        }
        if(!part)
          continue;
        const int n0 = (item - item0) * a.tile, n1 = min(n0 + a.tile, numnp);
        float *x32 = a.x32 + off, *r = a.r + off;
        const float *p = a.p + off, *ap = a.Ap + off;
        double rr = 0.0;
        for(int nb = n0 + t; nb < n1; nb += kU * (int)blockDim.x)
        {
          float pv[kU][3], av[kU][3], xv[kU][3], rv[kU][3], iv[kU][3];
#pragma unroll
          for(int u = 0; u < kU; u++)
          {
            const int n = nb + u * (int)blockDim.x;
            const bool in = n < n1;
#pragma unroll
            for(int c = 0; c < 3; c++)
            {
              const long id = (long)c * numnp + n;
              pv[u][c] = in ? __ldcg(p + id) : 0.0f;
              av[u][c] = in ? __ldcg(ap + id) : 0.0f;
              xv[u][c] = in ? __ldcg(x32 + id) : 0.0f;
              rv[u][c] = in ? __ldcg(r + id) : 0.0f;
              iv[u][c] = in ? __ldg(st.invd + id) : 0.0f;
            }
          }
#pragma unroll
          for(int u = 0; u < kU; u++)
          {
            const int n = nb + u * (int)blockDim.x;
            if(n >= n1)
              continue;
#pragma unroll
            for(int c = 0; c < 3; c++)
            {
              const long id = (long)c * numnp + n;
              x32[id] = fmaf(al, pv[u][c], xv[u][c]);
              const float ri = fmaf(-al, av[u][c], rv[u][c]);
              r[id] = ri;
              const float di = st.inv_theta * iv[u][c] * ri;
              st.x[id] = di;
              st.d[id] = di;
              rr += (double)ri * (double)ri;
            }
          }
        }
        double v[1] = {rr};
        block_sum<1>(v, sh);
        if(t == 0)
        {
          a.part[4L * item + 3] = v[0];
          if(item == item0)
            a.s[d].iter += 1;
        }
        __syncthreads();
      }
    }
    grid.sync();
    // ---- F: each design's own FP64 refresh request (r . r fell by the
    // factor `refresh` below the last FP64 residual, below the target, the
    // iteration cap, or not a number)
    {
      int cd = -1;
      for(int item = s0.i0; item < s0.i1; item++)
      {
        const int d = a.item_design[item];
        if(d == cd)
          continue;
        cd = d;
        const BatchDesign &D = a.des[d];
        if(item != D.item0 || !takes_part(a, d, 0))
          continue;
        const double rr = design_sum(a, D, 3, sh, bc);
        if(t == 0)
        {
          BScal &S = a.s[d];
          const bool fin = !(rr == rr) || S.iter >= S.maxit;
          const bool fresh = fin || rr < S.tol2 || rr < S.delta2 * S.rr_ref ||
                             S.iter - S.last_refresh >= kRefreshEvery;
          S.final_ = fin ? 1 : 0;
          S.refresh = fresh ? 1 : 0;
          if(fresh)
            atomicAdd(&a.ctl[1 + (it & 1)], 1);
        }
      }
      if(blockIdx.x == 0 && t == 0)
        a.ctl[1 + ((it + 1) & 1)] = 0; // the counter of the next iteration
    }
    grid.sync();
    // A refresh of some designs takes as long as one of all (each design's
    // node tiles are spread over many CTAs), so once one design asks, every
    // design refreshes: x += x32, x32 = 0, then r = b - K x in FP64
    if(*(volatile int *)&a.ctl[1 + (it & 1)] != 0)
    {
      // ---- R1: x += x32, x32 = 0; the designs that did not ask are marked
      // (refresh = 2) so that the stop test below knows the refresh was forced
      int cd = -1, numnp = 0, item0 = 0;
      long off = 0;
      bool part = false;
      double *x64 = nullptr;
      for(int item = s0.i0; item < s0.i1; item++)
      {
        const int d = a.item_design[item];
        if(d != cd)
        {
          cd = d;
          part = takes_part(a, d, 0);
          const BatchDesign &D = a.des[d];
          numnp = D.g.numnp;
          off = D.off;
          item0 = D.item0;
          x64 = D.x64;
        }
        if(!part)
          continue;
        if(item == item0 && t == 0 && a.s[d].refresh == 0)
          a.s[d].refresh = 2;
        const int n0 = (item - item0) * a.tile, n1 = min(n0 + a.tile, numnp);
        float *x32 = a.x32 + off;
        for(int nb = n0 + t; nb < n1; nb += kU * (int)blockDim.x)
        {
          float xv[kU][3];
          double yv[kU][3];
#pragma unroll
          for(int u = 0; u < kU; u++)
          {
            const int n = nb + u * (int)blockDim.x;
#pragma unroll
            for(int c = 0; c < 3; c++)
            {
              const long id = (long)c * numnp + n;
              xv[u][c] = n < n1 ? __ldcg(x32 + id) : 0.0f;
              yv[u][c] = n < n1 ? __ldcg(x64 + id) : 0.0;
            }
          }
#pragma unroll
          for(int u = 0; u < kU; u++)
          {
            const int n = nb + u * (int)blockDim.x;
            if(n < n1)
#pragma unroll
              for(int c = 0; c < 3; c++)
              {
                const long id = (long)c * numnp + n;
                x64[id] = yv[u][c] + (double)xv[u][c];
                x32[id] = 0.0f;
              }
          }
        }
      }
      grid.sync();
      // ---- R2: r = b - K x in FP64, partial r . r (slot 0), the first
      // smoothing step redone from this r
      for(int item = s0.i0; item < s0.i1; item++)
      {
        const int d = a.item_design[item];
        if(!takes_part(a, d, 0))
          continue;
        const BatchDesign &D = a.des[d];
        const BmDesign &B = m.bm[d];
        const int n0 = (item - D.item0) * a.tile;
        double rr = 0.0;
        // the FP64 node stencil leaves no registers to hold the design's
        // fields: they are read from the tables
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
            const float r32 = (float)ri;
            a.r[o] = r32;
            step0_of(B)(id, r32);
            rr += ri * ri;
          }
        }
        double v[1] = {rr};
        block_sum<1>(v, sh);
        if(t == 0)
          a.part[4L * item + 0] = v[0];
        __syncthreads();
      }
      grid.sync();
    }
    // ---- V: z = M r, partials z . r, z . Ap
    vcycle(0);
    // ---- P3: beta = -z.Ap / p.Ap, p = z + beta p; the design's first item
    // stores z . r and, after a refresh, takes the stop test on the FP64
    // residual
    {
      int cd = -1, numnp = 0, item0 = 0;
      long off = 0;
      bool part = false;
      double beta = 0.0;
      for(int item = s0.i0; item < s0.i1; item++)
      {
        const int d = a.item_design[item];
        if(d != cd)
        {
          cd = d;
          part = takes_part_block(a, d, 0, &part_flag);
          if(part)
          {
            const BatchDesign &D = a.des[d];
            const BmLevel &L0 = m.bm[d].lv[0];
            const double pap = range_sum(m.partc, L0.mitem0, L0.mitems, 0, sh, bc);
            const double zap = range_sum(m.partc, L0.mitem0, L0.mitems, 2, sh, bc);
            beta = -zap / pap;
            numnp = D.g.numnp;
            off = D.off;
            item0 = D.item0;
          }
        }
        if(!part)
          continue;
        if(item == item0)
        {
          const BatchDesign &D = a.des[d];
          const BmLevel &L0 = m.bm[d].lv[0];
          const double rz = range_sum(m.partc, L0.mitem0, L0.mitems, 1, sh, bc);
          const bool fresh = *(volatile const int *)&a.s[d].refresh != 0;
          const double rr = fresh ? design_sum(a, D, 0, sh, bc) : 0.0;
          if(t == 0)
          {
            BScal &S = a.s[d];
            S.rz = rz;
            if(fresh)
            {
              // stagnation is measured between the refreshes the design
              // asked for: a forced one may follow the last by one iteration
              if(S.refresh == 1)
              {
                S.nstall = rr > 0.81 * S.rr_nat ? S.nstall + 1 : 0;
                S.rr_nat = rr;
              }
              S.rr_true = S.rr_ref = rr;
              S.nrefresh += 1;
              S.last_refresh = S.iter;
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
            }
            if(!S.done && !(beta == beta && rz == rz))
            {
              S.done = 1;
              S.status = ICARAT_ERR_NAN;
            }
            if(S.done)
              atomicSub(&a.ctl[0], 1);
          }
        }
        const int n0 = (item - item0) * a.tile, n1 = min(n0 + a.tile, numnp);
        xpby_nodes(a.p + off, a.z + off, (float)beta, numnp, n0, n1);
      }
    }
    grid.sync();
  }
}

} // namespace icarat_b200
