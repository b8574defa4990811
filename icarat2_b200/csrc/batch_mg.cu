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
//   P1  Ap = K p (FP32 node stencil), partial p . Ap
//   P2  alpha; x32 += alpha p, r -= alpha Ap, partial r . r; and the first
//       Chebyshev step of the finest level from zero, x = d = D^-1 r / theta
//   V   z = M r: one V-cycle over all designs (per level down: deg-1
//       Chebyshev steps, residual, restriction fused with the next level's
//       first Chebyshev step; coarsest: y = W b, x = W^T y; per level up:
//       prolongation, deg Chebyshev steps; the finest level's last step
//       writes z with the partials z . r and z . Ap)
//   P3  beta = -z.Ap / p.Ap (flexible CG), p = z + beta p; the design's
//       first item decides an FP64 refresh
//   R   (designs that refresh) x += x32; r = b - K x in FP64; z = M r;
//       p = z (restart); stop test on the FP64 residual
// Vectors and the V-cycle are FP32 (as the mixed-precision solver's);
// the solution, right-hand side, dot products and scalars are FP64; the
// coarse dense solve is FP64.  Every grid barrier is reached by every CTA
// the same number of times; the loop is capped at maxit + 2 iterations.
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
// node column and z range of this thread in column item `item` of level Lv;
// false for the columns past the level's last
__device__ __forceinline__ bool col_item(const BmLevel &Lv, int item, int &i, int &j, int &k0,
                                         int &k1)
{
  const int q = item - Lv.mitem0;
  const int col = (q % Lv.ncb) * kBatchThreads + (int)threadIdx.x;
  k0 = (q / Lv.ncb) * Lv.kc;
  k1 = min(k0 + Lv.kc, Lv.g.NZ);
  if(col >= Lv.g.NX * Lv.g.NY)
    return false;
  i = col % Lv.g.NX;
  j = col / Lv.g.NX;
  return true;
}
} // namespace

__global__ void __launch_bounds__(kBatchThreads, 3) k_batch_mg(BatchArgs a, BmArgs m)
{
  cg::grid_group grid = cg::this_grid();
  __shared__ double sh[4 * 32];
  __shared__ double bc[4];
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

  // first Chebyshev step of the finest level from zero, fused into the
  // phases that produce r (node o of design D, component offset id)
  auto first_step0 = [&](const BmDesign &B, long id, float ri)
  {
    const float di = B.inv_theta * __ldg(B.lv[0].invd + id) * ri;
    B.lv[0].x[id] = di;
    B.lv[0].r[id] = di;
  };

  // one Chebyshev step on level l of the designs in `mode`:
  // d = c1 d + c2 D^-1 (b - K x), xo = x + d; on the finest level's last
  // step (fin) xo is z and the partials z . r (slot 1) and z . Ap (slot 2)
  // are written
  auto cheb = [&](int l, int mode, bool post, int k, bool fin)
  {
    const Span sp = span_of(m.lv_col_items[l]);
    const int c = cur[l];
    for(int item = sp.i0; item < sp.i1; item++)
    {
      const int d = m.lv_col_design[l][item];
      if(!takes_part(a, d, mode))
        continue;
      const BmDesign &B = m.bm[d];
      const BmLevel &Lv = B.lv[l];
      const BatchDesign &D = a.des[d];
      const float c1 = post ? B.post_c1[k] : B.pre_c1[k];
      const float c2 = post ? B.post_c2[k] : B.pre_c2[k];
      const float *x = c ? Lv.t : Lv.x;
      float *xo = fin ? a.z + D.off : (c ? Lv.x : Lv.t);
      const float *b = l == 0 ? a.r + D.off : Lv.b;
      double rz = 0.0, zap = 0.0;
      int i, j, k0, k1;
      if(col_item(Lv, item, i, j, k0, k1))
        column_Ku<float, KeParamF, true>(
            Lv.g, a.kef, Lv.E32, x, i, j, k0, k1,
            [&](int kk, const float(&acc)[3], const float(&uc)[3])
            {
              const int n = i + j * Lv.g.NX + kk * Lv.g.NX * Lv.g.NY;
              const unsigned f = Lv.fix[n];
#pragma unroll
              for(int q = 0; q < 3; q++)
              {
                const long id = (long)q * Lv.g.numnp + n;
                float dn = 0.0f;
                if(!((f >> q) & 1u))
                  dn = (c1 != 0.0f ? c1 * __ldcg(Lv.r + id) : 0.0f) +
                       c2 * __ldg(Lv.invd + id) * (__ldcg(b + id) - acc[q]);
                Lv.r[id] = dn;
                const float xn = uc[q] + dn;
                xo[id] = xn;
                if(fin)
                {
                  rz += (double)xn * (double)__ldcg(b + id);
                  zap += (double)xn * (double)__ldcg(a.Ap + D.off + id);
                }
              }
            });
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
    for(int item = sp.i0; item < sp.i1; item++)
    {
      const int d = m.lv_col_design[l][item];
      if(!takes_part(a, d, mode))
        continue;
      const BmDesign &B = m.bm[d];
      const BmLevel &Lv = B.lv[l];
      const float *x = c ? Lv.t : Lv.x;
      const float *b = l == 0 ? a.r + a.des[d].off : Lv.b;
      int i, j, k0, k1;
      if(col_item(Lv, item, i, j, k0, k1))
        column_Ku<float, KeParamF, true>(
            Lv.g, a.kef, Lv.E32, x, i, j, k0, k1,
            [&](int kk, const float(&acc)[3], const float(&)[3])
            {
              const int n = i + j * Lv.g.NX + kk * Lv.g.NX * Lv.g.NY;
              const unsigned f = Lv.fix[n];
#pragma unroll
              for(int q = 0; q < 3; q++)
              {
                const long id = (long)q * Lv.g.numnp + n;
                Lv.r[id] = ((f >> q) & 1u) ? 0.0f : __ldcg(b + id) - acc[q];
              }
            });
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
      const int n0 = (item - C.item0) * a.tile, n1 = min(n0 + a.tile, C.g.numnp);
      for(int n = n0 + t; n < n1; n += blockDim.x)
      {
        float sr[3];
        restrict_node<float, true>(F.g, C.g, F.r, n, sr);
        const unsigned fx = C.fix[n];
#pragma unroll
        for(int q = 0; q < 3; q++)
        {
          const long id = (long)q * C.g.numnp + n;
          const float bq = ((fx >> q) & 1u) ? 0.0f : sr[q];
          C.b[id] = bq;
          if(!smooth)
          {
            // coarsest level: the dense solve's right-hand side, gathered
            const int u = __ldg(B.cmap + 3L * n + q);
            if(u >= 0)
              B.v[u] = (double)bq;
          }
          else
          {
            const float di = B.inv_theta * __ldg(C.invd + id) * bq;
            C.x[id] = di;
            C.r[id] = di;
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
      const BmLevel &C = B.lv[L - 1];
      const int q = item - B.citem0;
      const int r0 = q * m.ctile, r1 = min(r0 + m.ctile, B.nc);
      for(int r = r0 + warp; r < r1; r += nw)
      {
        // four independent partial sums: four loads of the row and of v in
        // flight per lane
        const double *row = B.W + (long)r * B.nc;
        double s4[4] = {0.0, 0.0, 0.0, 0.0};
        int j = lane;
        for(; j + 96 <= r; j += 128)
#pragma unroll
          for(int u = 0; u < 4; u++)
            s4[u] = fma(__ldg(row + j + 32 * u), __ldcg(B.v + j + 32 * u), s4[u]);
        for(; j <= r; j += 32)
          s4[0] = fma(__ldg(row + j), __ldcg(B.v + j), s4[0]);
        double sum = (s4[0] + s4[1]) + (s4[2] + s4[3]);
        for(int o = 16; o > 0; o >>= 1)
          sum += __shfl_xor_sync(0xffffffffu, sum, o);
        if(lane == 0)
          B.y[r] = sum;
      }
      // this item's share of the coarsest iterate, cleared (constrained
      // entries stay 0; the free ones are written below)
      const long nv = 3L * C.g.numnp;
      const long per = (nv + B.citems - 1) / B.citems;
      const long e0 = (long)q * per, e1 = min(e0 + per, nv);
      for(long e = e0 + t; e < e1; e += blockDim.x)
        C.x[e] = 0.0f;
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
      const BmLevel &C = B.lv[L - 1];
      const int q = item - B.citem0;
      const int r0 = q * m.ctile, r1 = min(r0 + m.ctile, B.nc);
      for(int r = r0 + warp; r < r1; r += nw)
      {
        const double *row = B.WT + (long)r * B.nc;
        double s4[4] = {0.0, 0.0, 0.0, 0.0};
        int j = r + lane;
        for(; j + 96 < B.nc; j += 128)
#pragma unroll
          for(int u = 0; u < 4; u++)
            s4[u] = fma(__ldg(row + j + 32 * u), __ldcg(B.y + j + 32 * u), s4[u]);
        for(; j < B.nc; j += 32)
          s4[0] = fma(__ldg(row + j), __ldcg(B.y + j), s4[0]);
        double sum = (s4[0] + s4[1]) + (s4[2] + s4[3]);
        for(int o = 16; o > 0; o >>= 1)
          sum += __shfl_xor_sync(0xffffffffu, sum, o);
        if(lane == 0)
          C.x[__ldg(B.map + r)] = (float)sum;
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
      float *x = c ? F.t : F.x;
      const float *xc = cc ? C.t : C.x;
      const int n0 = (item - F.item0) * a.tile, n1 = min(n0 + a.tile, F.g.numnp);
      for(int n = n0 + t; n < n1; n += blockDim.x)
      {
        float s[3];
        prolong_node<float, true>(F.g, C.g, xc, n, s);
        const unsigned fx = F.fix[n];
#pragma unroll
        for(int q = 0; q < 3; q++)
          if(!((fx >> q) & 1u))
          {
            const long id = (long)q * F.g.numnp + n;
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
        first_step0(B, id, ri);
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
      S.rr_ref = S.rr_true = bb;
      S.tol2 = a.tol * a.tol * bb;
      S.delta2 = a.delta * a.delta;
      S.iter = 0;
      S.maxit = a.maxit;
      S.refresh = S.final_ = S.nrefresh = S.nstall = 0;
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
  for(int item = s0.i0; item < s0.i1; item++)
  {
    const int d = a.item_design[item];
    if(!takes_part(a, d, 0))
      continue;
    const BatchDesign &D = a.des[d];
    const BmLevel &L0 = m.bm[d].lv[0];
    const double rz = range_sum(m.partc, L0.mitem0, L0.mitems, 1, sh, bc);
    const int n0 = (item - D.item0) * a.tile;
    for(int n = n0 + t; n < min(n0 + a.tile, D.g.numnp); n += blockDim.x)
#pragma unroll
      for(int c = 0; c < 3; c++)
      {
        const long o = D.off + (long)c * D.g.numnp + n;
        a.p[o] = __ldcg(a.z + o);
      }
    if(item == D.item0 && t == 0)
      a.s[d].rz = rz;
  }
  grid.sync();

  for(int it = 0; it < a.maxit + 2; it++)
  {
    if(*(volatile int *)&a.ctl[0] <= 0)
      break;
    // ---- P1: Ap = K p, partial p . Ap (finest-level column items)
    {
      const Span sp = span_of(m.lv_col_items[0]);
      for(int item = sp.i0; item < sp.i1; item++)
      {
        const int d = m.lv_col_design[0][item];
        if(!takes_part(a, d, 0))
          continue;
        const BatchDesign &D = a.des[d];
        const BmLevel &Lv = m.bm[d].lv[0];
        double pap = 0.0;
        int i, j, k0, k1;
        if(col_item(Lv, item, i, j, k0, k1))
          column_Ku<float, KeParamF, true>(
              D.g, a.kef, D.E32, a.p + D.off, i, j, k0, k1,
              [&](int kk, const float(&acc)[3], const float(&uc)[3])
              {
                const int n = i + j * D.g.NX + kk * D.g.NX * D.g.NY;
                const unsigned f = D.fix[n];
#pragma unroll
                for(int c = 0; c < 3; c++)
                {
                  const float y = ((f >> c) & 1u) ? 0.0f : acc[c];
                  a.Ap[D.off + (long)c * D.g.numnp + n] = y;
                  pap += (double)uc[c] * (double)y;
                }
              });
        double v[1] = {pap};
        block_sum<1>(v, sh);
        if(t == 0)
          m.partc[4L * item] = v[0];
        __syncthreads();
      }
    }
    grid.sync();
    // ---- P2: x32, r updates, partial r . r, first smoothing step
    {
      int cached = -1;
      double alpha = 0.0;
      for(int item = s0.i0; item < s0.i1; item++)
      {
        const int d = a.item_design[item];
        if(!takes_part(a, d, 0))
          continue;
        const BatchDesign &D = a.des[d];
        const BmDesign &B = m.bm[d];
        if(d != cached)
        {
          const double pap =
              range_sum(m.partc, B.lv[0].mitem0, B.lv[0].mitems, 0, sh, bc);
          alpha = a.s[d].rz / pap;
          cached = d;
        }
        const float al = (float)alpha;
        const int n0 = (item - D.item0) * a.tile;
        double rr = 0.0;
        for(int n = n0 + t; n < min(n0 + a.tile, D.g.numnp); n += blockDim.x)
#pragma unroll
          for(int c = 0; c < 3; c++)
          {
            const long id = (long)c * D.g.numnp + n, o = D.off + id;
            const float pi = __ldcg(a.p + o), api = __ldcg(a.Ap + o);
            a.x32[o] = fmaf(al, pi, __ldcg(a.x32 + o));
            const float ri = fmaf(-al, api, __ldcg(a.r + o));
            a.r[o] = ri;
            first_step0(B, id, ri);
            rr += (double)ri * (double)ri;
          }
        double v[1] = {rr};
        block_sum<1>(v, sh);
        if(t == 0)
        {
          a.part[4L * item + 3] = v[0];
          if(item == D.item0)
            a.s[d].iter += 1;
        }
        __syncthreads();
      }
    }
    grid.sync();
    // ---- V: z = M r, partials z . r, z . Ap
    vcycle(0);
    // ---- P3: p = z + beta p; refresh decision
    {
      int cached = -1;
      double beta = 0.0;
      for(int item = s0.i0; item < s0.i1; item++)
      {
        const int d = a.item_design[item];
        if(!takes_part(a, d, 0))
          continue;
        const BatchDesign &D = a.des[d];
        if(d != cached)
        {
          const BmLevel &L0 = m.bm[d].lv[0];
          const double pap = range_sum(m.partc, L0.mitem0, L0.mitems, 0, sh, bc);
          const double zap = range_sum(m.partc, L0.mitem0, L0.mitems, 2, sh, bc);
          beta = -zap / pap;
          cached = d;
          if(item == D.item0)
          {
            const double rz = range_sum(m.partc, L0.mitem0, L0.mitems, 1, sh, bc);
            const double rr = design_sum(a, D, 3, sh, bc);
            if(t == 0)
            {
              BScal &S = a.s[d];
              S.rz = rz;
              const bool nan = !(rr == rr) || !(beta == beta);
              S.final_ = (nan || S.iter >= S.maxit) ? 1 : 0;
              S.refresh = (S.final_ || rr < S.tol2 || rr < S.delta2 * S.rr_ref) ? 1 : 0;
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
            a.p[o] = fmaf(be, __ldcg(a.p + o), __ldcg(a.z + o));
          }
      }
      if(blockIdx.x == 0 && t == 0)
        a.ctl[1 + ((it + 1) & 1)] = 0; // the counter of the next iteration
    }
    grid.sync();
    if(*(volatile int *)&a.ctl[1 + (it & 1)] == 0)
      continue;
    // ---- R1: x += x32, x32 = 0 for the designs that refresh
    for(int item = s0.i0; item < s0.i1; item++)
    {
      const int d = a.item_design[item];
      if(!takes_part(a, d, 1))
        continue;
      const BatchDesign &D = a.des[d];
      const int n0 = (item - D.item0) * a.tile;
      for(int n = n0 + t; n < min(n0 + a.tile, D.g.numnp); n += blockDim.x)
#pragma unroll
        for(int c = 0; c < 3; c++)
        {
          const long id = (long)c * D.g.numnp + n;
          D.x64[id] += (double)__ldcg(a.x32 + D.off + id);
          a.x32[D.off + id] = 0.0f;
        }
    }
    grid.sync();
    // ---- R2: r = b - K x in FP64; partial r . r (slot 0); first smoothing step
    for(int item = s0.i0; item < s0.i1; item++)
    {
      const int d = a.item_design[item];
      if(!takes_part(a, d, 1))
        continue;
      const BatchDesign &D = a.des[d];
      const BmDesign &B = m.bm[d];
      const int n0 = (item - D.item0) * a.tile;
      double rr = 0.0;
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
          first_step0(B, id, r32);
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
    // ---- z = M r for the refreshing designs
    vcycle(1);
    // ---- R3: p = z (restart), stop test on the FP64 residual
    for(int item = s0.i0; item < s0.i1; item++)
    {
      const int d = a.item_design[item];
      if(!takes_part(a, d, 1))
        continue;
      const BatchDesign &D = a.des[d];
      const int n0 = (item - D.item0) * a.tile;
      for(int n = n0 + t; n < min(n0 + a.tile, D.g.numnp); n += blockDim.x)
#pragma unroll
        for(int c = 0; c < 3; c++)
        {
          const long o = D.off + (long)c * D.g.numnp + n;
          a.p[o] = __ldcg(a.z + o);
        }
      if(item != D.item0)
        continue;
      const double rr = design_sum(a, D, 0, sh, bc);
      const BmLevel &L0 = m.bm[d].lv[0];
      const double rz = range_sum(m.partc, L0.mitem0, L0.mitems, 1, sh, bc);
      if(t == 0)
      {
        BScal &S = a.s[d];
        S.nstall = rr > 0.81 * S.rr_true ? S.nstall + 1 : 0;
        S.rr_true = S.rr_ref = rr;
        S.rz = rz;
        S.nrefresh += 1;
        // S.refresh stays set until the next P3 decides anew: the other
        // items of this design test it in this same phase
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
