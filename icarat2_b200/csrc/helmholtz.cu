// Helmholtz PDE density filter (FilterHelmholtz<E,N>,
// src/optimization/filter_helm.hpp) on the voxel grid.
//
// The reference assembles, per element and Gauss point (makeKeFint,
// :179-223), Ke += (N N^T + B^T (R / (2 sqrt 3))^2 I B) jac and
// fe += s N jac (fe /= ipmax for the sensitivity call), solves the nodal
// scalar system K val = F with "Eigen_CG" (a Jacobi-preconditioned CG,
// solvers.cpp:63-91, tolerance 1e-10 and 10000 iterations by default,
// solvers.hpp:89-90) and maps back per element (divideToElement, :225-257):
// out = sum_gp N . val_e, divided by ipmax for the density call.
//
// On the uniform voxel box every element has the same 8 x 8 matrix, so the
// assembled K is a 27-point node stencil whose coefficients depend only on
// which of the node's 8 neighbouring elements exist: 3 x 3 x 3 node classes
// (lower face, interior, upper face per axis).  The table of 27 classes x 27
// neighbour slots is assembled once on the host in the reference's order
// (ascending element id) for the Jacobi diagonal; the solve runs
// matrix-free with the same operator in sum-factorised form (k_helm_spmv).
// The CG iteration
// keeps the device-resident scalar logic of the elasticity solve (one
// stop-flag read per graph replay of `kHelmChunk` iterations).
#include <cmath>

#include "internal.cuh"

namespace icarat_b200
{

// the CG start of pcg.cu
__global__ void k_cg_init(int n, const double *__restrict__ b,
                          const double *__restrict__ invd, double *__restrict__ x,
                          double *__restrict__ r, double *__restrict__ z,
                          double *__restrict__ p, double *__restrict__ partials,
                          CgScalars *s, double tol, int maxit, int jacobi);

namespace
{

constexpr int kHelmChunk = 16;
constexpr int kHelmThreads = 256;
constexpr int kHelmClasses = 27;

struct HelmGrid
{
  int nx, ny, nz, NX, NY, numnp, nelx;
};

// integrals of the shape functions over the element: sum_gp N_a jac (the
// right-hand side weights) and sum_gp N_a (the readout weights); corners in
// bit order a = ax + 2 ay + 4 az
struct HelmWeights
{
  double nj[8], ns[8];
};

HelmGrid hgrid(const icarat_ctx *c)
{
  return HelmGrid{c->nx, c->ny, c->nz, c->NX, c->NY, c->numnp, c->nelx};
}

__device__ __forceinline__ int node_class(int i, int n)
{
  return i == 0 ? 0 : (i == n - 1 ? 2 : 1);
}

// F = sum over the node's elements of s_e nj[a] (/8 for the sensitivity
// call), elements in ascending id like the reference's assembly
__global__ void k_helm_rhs(HelmGrid g, HelmWeights w, const double *__restrict__ in,
                           double *__restrict__ F, int sens)
{
  for(int n = blockIdx.x * blockDim.x + threadIdx.x; n < g.numnp;
      n += gridDim.x * blockDim.x)
  {
    const int i = n % g.NX, rest = n / g.NX, j = rest % g.NY, k = rest / g.NY;
    double f = 0.0;
    for(int oz = -1; oz <= 0; oz++)
      for(int oy = -1; oy <= 0; oy++)
        for(int ox = -1; ox <= 0; ox++)
        {
          const int ei = i + ox, ej = j + oy, ek = k + oz;
          if(ei < 0 || ei >= g.nx || ej < 0 || ej >= g.ny || ek < 0 || ek >= g.nz)
            continue;
          const int a = -ox - 2 * oy - 4 * oz;
          double fe = __dmul_rn(__ldg(in + ei + (long)ej * g.nx + (long)ek * g.nx * g.ny),
                                w.nj[a]);
          if(sens)
            fe = __ddiv_rn(fe, 8.0);
          f = __dadd_rn(f, fe);
        }
    F[n] = f;
  }
}

// inverse of the stencil's centre coefficient (the Jacobi preconditioner)
__global__ void k_helm_invd(HelmGrid g, const double *__restrict__ coef,
                            double *__restrict__ invd)
{
  for(int n = blockIdx.x * blockDim.x + threadIdx.x; n < g.numnp;
      n += gridDim.x * blockDim.x)
  {
    const int i = n % g.NX, rest = n / g.NX, j = rest % g.NY, k = rest / g.NY;
    const int NZ = g.nz + 1;
    const int cls = node_class(i, g.NX) + 3 * node_class(j, g.NY) + 9 * node_class(k, NZ);
    invd[n] = 1.0 / coef[27 * cls + 13];
  }
}

// Ap = K p and alpha = zr / (p . Ap), by sum factorisation.
//
// With trilinear shape functions and exact 2-point Gauss rules the element
// matrix is a tensor product, Ke = Mx (x) My (x) Mz + c (Sx (x) My (x) Mz +
// Mx (x) Sy (x) Mz + Mx (x) My (x) Sz), c = (R / (2 sqrt 3))^2, with the 1-D
// element mass h/6 [2 1; 1 2] and stiffness 1/h [1 -1; -1 1]; assembled on
// the box it stays one, with the 3-point 1-D stencils m, s of each node
// class (lower face, inside, upper face).  So every plane of p contributes
// through two in-plane sums per node, A = (mx my + c (sx my + mx sy)) p and
// B = mx my p, and Ap(k) = sum_dz mz A(k+dz) + c sz B(k+dz).
//
// A block of 8 warps owns 32 x 8 kHelmRows node columns (a warp kHelmRows
// rows of 32 nodes along x) and marches through kHelmTz planes, holding A
// and B of planes k-1, k, k+1 in registers.  The planes of p come through
// shared memory: a ring of kHelmDepth halo tiles filled by cp.async,
// kHelmDepth - 1 planes ahead of the plane being reduced, so later planes
// are in flight without holding registers.  Positions outside the box are
// stored as 0 (their stencil weights are 0 as well).  Measured on the B200
// at 257 x 129 x 129 nodes: about 50 us per launch, like a variant with a
// one-plane register lookahead and one with two rows per thread; the limit
// is dependent-latency (FP64 FMA chains, barriers), not DRAM.
constexpr int kHelmTx = 32, kHelmWarps = 8, kHelmRows = 1, kHelmTz = 16, kHelmDepth = 4;
constexpr int kHelmTy = kHelmWarps * kHelmRows;
constexpr int kHaloX = kHelmTx + 2, kHaloY = kHelmTy + 2, kHalo = kHaloX * kHaloY;
constexpr int kStage = (kHalo + kHelmTx * kHelmWarps - 1) / (kHelmTx * kHelmWarps);

// 1-D stencils [axis][class][d + 1] and the diffusion coefficient c
struct HelmAxes
{
  double m[3][3][3], s[3][3][3];
  double c;
};

// 8-byte global -> shared copies (cp.async), one commit group per staged
// plane, and a wait for all but the newest kHelmDepth - 1 groups
__device__ __forceinline__ void cp_async8(double *dst, const double *src)
{
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit()
{
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}
__device__ __forceinline__ void cp_async_wait_ring()
{
  asm volatile("cp.async.wait_group %0;\n" ::"n"(kHelmDepth - 1) : "memory");
}

// this thread's staged halo positions: in-plane offset (or -1 outside)
struct HelmStage
{
  long off[kStage];
};

// halo tile of plane kk (rows j0-1 .. j0+kHelmTy, columns i0-1 .. i0+32)
// into buf; one commit group per call, empty when the plane is not needed
__device__ __forceinline__ void helm_stage(double *buf, const double *__restrict__ p,
                                          const HelmStage &st, int NZ, long plane, int kk,
                                          bool needed)
{
  if(needed)
  {
    const bool inz = kk >= 0 && kk < NZ;
#pragma unroll
    for(int q = 0; q < kStage; q++)
    {
      const int e = threadIdx.x + q * kHelmTx * kHelmWarps;
      if(e < kHalo)
      {
        if(inz && st.off[q] >= 0)
          cp_async8(buf + e, p + st.off[q] + kk * plane);
        else
          buf[e] = 0.0;
      }
    }
  }
  cp_async_commit();
}

__global__ void __launch_bounds__(kHelmTx * kHelmWarps)
    k_helm_spmv(HelmGrid g, HelmAxes ax, const double *__restrict__ p,
                double *__restrict__ Ap, double *__restrict__ partials, CgScalars *s)
{
  chain_wait();
  __shared__ double ring[kHelmDepth][kHalo];
  __shared__ double sh[64];
  if(s->done)
    return;
  const int NZ = g.nz + 1;
  const long plane = (long)g.NX * g.NY;
  const int tiles_x = (g.NX + kHelmTx - 1) / kHelmTx, tiles_y = (g.NY + kHelmTy - 1) / kHelmTy;
  const int tiles = tiles_x * tiles_y * ((NZ + kHelmTz - 1) / kHelmTz);
  const double c = ax.c;
  const int lx = threadIdx.x & 31, ly = (threadIdx.x >> 5) * kHelmRows;
  double dot = 0.0;
  for(int t = blockIdx.x; t < tiles; t += gridDim.x)
  {
    const int i0 = (t % tiles_x) * kHelmTx, j0 = (t / tiles_x % tiles_y) * kHelmTy;
    const int k0 = t / (tiles_x * tiles_y) * kHelmTz;
    const int k1 = min(k0 + kHelmTz, NZ);
    const int i = i0 + lx;
    HelmStage st;
#pragma unroll
    for(int q = 0; q < kStage; q++)
    {
      const int e = threadIdx.x + q * kHelmTx * kHelmWarps;
      const int x = i0 - 1 + e % kHaloX, y = j0 - 1 + e / kHaloX;
      st.off[q] = (x >= 0 && x < g.NX && y >= 0 && y < g.NY) ? x + (long)y * g.NX : -1;
    }
    double mx[3], sx[3], my[kHelmRows][3], sy[kHelmRows][3];
    const int cx = node_class(min(i, g.NX - 1), g.NX);
#pragma unroll
    for(int d = 0; d < 3; d++)
    {
      mx[d] = ax.m[0][cx][d];
      sx[d] = ax.s[0][cx][d];
    }
#pragma unroll
    for(int r = 0; r < kHelmRows; r++)
    {
      const int cy = node_class(min(j0 + ly + r, g.NY - 1), g.NY);
#pragma unroll
      for(int d = 0; d < 3; d++)
      {
        my[r][d] = ax.m[1][cy][d];
        sy[r][d] = ax.s[1][cy][d];
      }
    }
    // planes k0-1 .. k1 are reduced, plane m in ring slot (m - k0 + 1) % depth;
    // the ring of the previous tile is no longer read past this barrier, and
    // every copy of that tile has landed (its groups past plane k1 were empty)
    __syncthreads();
#pragma unroll
    for(int q = 0; q < kHelmDepth; q++)
      helm_stage(ring[q], p, st, NZ, plane, k0 - 1 + q, k0 - 1 + q <= k1);
    double A0[kHelmRows], B0[kHelmRows], A1[kHelmRows], B1[kHelmRows], A2[kHelmRows],
        B2[kHelmRows], P1[kHelmRows], P2[kHelmRows];
    for(int m = k0 - 1; m <= k1; m++)
    {
      const int slot = (m - k0 + 1) % kHelmDepth;
      cp_async_wait_ring();
      __syncthreads();
      {
        const double *buf = ring[slot] + ly * kHaloX + lx;
        double rm[kHelmRows + 2], rs[kHelmRows + 2];
#pragma unroll
        for(int q = 0; q < kHelmRows + 2; q++)
        {
          const double vl = buf[q * kHaloX], v0 = buf[q * kHaloX + 1], vr = buf[q * kHaloX + 2];
          rm[q] = mx[0] * vl + mx[1] * v0 + mx[2] * vr;
          rs[q] = sx[0] * vl + sx[1] * v0 + sx[2] * vr;
          if(q >= 1 && q <= kHelmRows)
            P2[q - 1] = v0;
        }
#pragma unroll
        for(int r = 0; r < kHelmRows; r++)
        {
          const double pm = my[r][0] * rm[r] + my[r][1] * rm[r + 1] + my[r][2] * rm[r + 2];
          const double ps = my[r][0] * rs[r] + my[r][1] * rs[r + 1] + my[r][2] * rs[r + 2] +
                            sy[r][0] * rm[r] + sy[r][1] * rm[r + 1] + sy[r][2] * rm[r + 2];
          A2[r] = pm + c * ps;
          B2[r] = pm;
        }
      }
      __syncthreads(); // every thread has read the slot: refill it
      helm_stage(ring[slot], p, st, NZ, plane, m + kHelmDepth, m + kHelmDepth <= k1);
      if(m >= k0 + 1)
      {
        // output plane k = m - 1 from planes k-1, k, k+1
        const int k = m - 1;
        const int cz = node_class(k, NZ);
        const double mz0 = ax.m[2][cz][0], mz1 = ax.m[2][cz][1], mz2 = ax.m[2][cz][2];
        const double sz0 = ax.s[2][cz][0], sz1 = ax.s[2][cz][1], sz2 = ax.s[2][cz][2];
#pragma unroll
        for(int r = 0; r < kHelmRows; r++)
        {
          const double y = mz0 * A0[r] + mz1 * A1[r] + mz2 * A2[r] +
                           c * (sz0 * B0[r] + sz1 * B1[r] + sz2 * B2[r]);
          const int j = j0 + ly + r;
          if(i < g.NX && j < g.NY)
          {
            Ap[i + (long)j * g.NX + (long)k * plane] = y;
            dot += P1[r] * y;
          }
        }
      }
#pragma unroll
      for(int r = 0; r < kHelmRows; r++)
      {
        A0[r] = A1[r];
        B0[r] = B1[r];
        A1[r] = A2[r];
        B1[r] = B2[r];
        P1[r] = P2[r];
      }
    }
  }
  double v[1] = {dot};
  block_sum<1>(v, sh);
  if(threadIdx.x == 0)
    partials[blockIdx.x] = v[0];
  if(last_block(&s->counter))
  {
    double t[1];
    sum_partials<1>(partials, gridDim.x, t, sh);
    if(threadIdx.x == 0)
    {
      s->pAp = t[0];
      s->alpha = s->zr / t[0];
      s->counter = 0;
    }
  }
}

// Jacobi inverse diagonal per node class (27 values, 1 / centre coefficient
// of the class row)
struct HelmInvd
{
  double v[kHelmClasses];
};

__device__ __forceinline__ int helm_class(const HelmGrid &g, int n)
{
  const int i = n % g.NX, rest = n / g.NX, j = rest % g.NY, k = rest / g.NY;
  return node_class(i, g.NX) + 3 * node_class(j, g.NY) + 9 * node_class(k, g.nz + 1);
}

// The Jacobi CG update of k_cg_update_jacobi (x += alpha p, r -= alpha Ap,
// z = D^-1 r, beta, stop test) with D^-1 taken from the node's class instead
// of a vector and z not stored: k_helm_pupdate forms it again from r, with
// the same operations, so the iterates are those of the generic kernels on
// 16 bytes per node less.
__global__ void k_helm_update(HelmGrid g, HelmInvd iv, double *__restrict__ x,
                              double *__restrict__ r, const double *__restrict__ p,
                              const double *__restrict__ Ap, double *__restrict__ partials,
                              CgScalars *s)
{
  chain_wait();
  __shared__ double sh[64];
  if(s->done)
    return;
  const double alpha = s->alpha;
  double zr = 0.0, rr = 0.0;
  for(int n = blockIdx.x * blockDim.x + threadIdx.x; n < g.numnp;
      n += gridDim.x * blockDim.x)
  {
    x[n] += alpha * p[n];
    const double ri = r[n] - alpha * Ap[n];
    r[n] = ri;
    const double zi = ri * iv.v[helm_class(g, n)];
    zr += zi * ri;
    rr += ri * ri;
  }
  double v[2] = {zr, rr};
  block_sum<2>(v, sh);
  if(threadIdx.x == 0)
  {
    partials[blockIdx.x] = v[0];
    partials[gridDim.x + blockIdx.x] = v[1];
  }
  if(last_block(&s->counter))
  {
    double t[2];
    sum_partials<2>(partials, gridDim.x, t, sh);
    if(threadIdx.x == 0)
    {
      s->zr_new = t[0];
      s->beta = t[0] / s->zr;
      s->zr = t[0];
      cg_check(s, t[1]);
      s->counter = 0;
    }
  }
}

// p = z + beta p with z = D^-1 r
__global__ void k_helm_pupdate(HelmGrid g, HelmInvd iv, const double *__restrict__ r,
                               double *__restrict__ p, const CgScalars *s)
{
  chain_wait();
  if(s->done)
    return;
  const double beta = s->beta;
  for(int n = blockIdx.x * blockDim.x + threadIdx.x; n < g.numnp;
      n += gridDim.x * blockDim.x)
    p[n] = beta * p[n] + r[n] * iv.v[helm_class(g, n)];
}

// out_e = sum_a ns[a] val[node_a] (/8 for the density call)
__global__ void k_helm_out(HelmGrid g, HelmWeights w, const double *__restrict__ val,
                           double *__restrict__ out, int sens)
{
  const long plane = (long)g.NX * g.NY;
  for(int e = blockIdx.x * blockDim.x + threadIdx.x; e < g.nelx;
      e += gridDim.x * blockDim.x)
  {
    const int i = e % g.nx, j = (e / g.nx) % g.ny, k = e / (g.nx * g.ny);
    const long n0 = i + (long)j * g.NX + k * plane;
    double s = 0.0;
#pragma unroll
    for(int a = 0; a < 8; a++)
    {
      const long m = n0 + (a & 1) + ((a >> 1) & 1) * (long)g.NX + ((a >> 2) & 1) * plane;
      s = __dadd_rn(s, __dmul_rn(w.ns[a], __ldg(val + m)));
    }
    out[e] = sens ? s : __ddiv_rn(s, 8.0);
  }
}

int blocks_for(long n, int threads, int cap)
{
  long b = (n + threads - 1) / threads;
  if(b > cap)
    b = cap;
  return b < 1 ? 1 : (int)b;
}

} // namespace

// The 8 x 8 element matrix of one hx x hy x hz voxel and its shape-function
// integrals, 2 x 2 x 2 Gauss points (makeKeFint, filter_helm.hpp:203-217).
// The voxel's Jacobian is diag(hx, hy, hz) / 2.
void helm_element(double hx, double hy, double hz, double R, double *ke, double *nj,
                  double *ns)
{
  const double g = 1.0 / std::sqrt(3.0);
  const double cdiff = std::pow(R / (2.0 * std::sqrt(3.0)), 2);
  const double h[3] = {hx, hy, hz};
  const double jac = (hx * 0.5) * (hy * 0.5) * (hz * 0.5);
  for(int t = 0; t < 64; t++)
    ke[t] = 0.0;
  for(int a = 0; a < 8; a++)
    nj[a] = ns[a] = 0.0;
  for(int ip = 0; ip < 8; ip++)
  {
    const double r[3] = {(ip & 1) ? g : -g, (ip & 2) ? g : -g, (ip & 4) ? g : -g};
    double N[8], B[3][8];
    for(int a = 0; a < 8; a++)
    {
      double f[3], df[3];
      for(int d = 0; d < 3; d++)
      {
        const double sgn = ((a >> d) & 1) ? 1.0 : -1.0;
        f[d] = 1.0 + sgn * r[d];
        df[d] = sgn;
      }
      N[a] = 0.125 * f[0] * f[1] * f[2];
      B[0][a] = 0.125 * df[0] * f[1] * f[2] * (2.0 / h[0]);
      B[1][a] = 0.125 * f[0] * df[1] * f[2] * (2.0 / h[1]);
      B[2][a] = 0.125 * f[0] * f[1] * df[2] * (2.0 / h[2]);
    }
    for(int a = 0; a < 8; a++)
    {
      for(int b = 0; b < 8; b++)
      {
        double sb = 0.0;
        for(int d = 0; d < 3; d++)
          sb += B[d][a] * cdiff * B[d][b];
        ke[8 * a + b] += (N[a] * N[b] + sb) * jac;
      }
      nj[a] += N[a] * jac;
      ns[a] += N[a];
    }
  }
}

// 27 node classes x 27 neighbour slots: class (cx, cy, cz), c = 0 on the
// lower face, 1 inside, 2 on the upper face of an axis; the node's elements
// sit at offsets o in {-1, 0}^3 (o = -1 exists unless c = 0, o = 0 unless
// c = 2) and are summed in ascending element id like the assembly of
// setFromTriplets over the reference's element loop.
static void helm_class_table(const double *ke, double *coef)
{
  for(int cz = 0; cz < 3; cz++)
    for(int cy = 0; cy < 3; cy++)
      for(int cx = 0; cx < 3; cx++)
      {
        const int cls = cx + 3 * cy + 9 * cz;
        const int cc[3] = {cx, cy, cz};
        for(int q = 0; q < 27; q++)
        {
          const int dd[3] = {q % 3 - 1, q / 3 % 3 - 1, q / 9 - 1};
          double v = 0.0;
          for(int oz = -1; oz <= 0; oz++)
            for(int oy = -1; oy <= 0; oy++)
              for(int ox = -1; ox <= 0; ox++)
              {
                const int o[3] = {ox, oy, oz};
                bool ok = true;
                int a = 0, b = 0;
                for(int d = 0; d < 3; d++)
                {
                  if((o[d] == -1 && cc[d] == 0) || (o[d] == 0 && cc[d] == 2))
                    ok = false;
                  const int ad = -o[d], bd = ad + dd[d];
                  if(bd < 0 || bd > 1)
                    ok = false;
                  a |= ad << d;
                  b |= (bd & 1) << d;
                }
                if(ok)
                  v += ke[8 * a + b];
              }
          coef[27 * cls + q] = v;
        }
      }
}

// the assembled 1-D stencils of each axis: element mass h/6 [2 1; 1 2] and
// stiffness 1/h [1 -1; -1 1] summed over the one (face) or two (inside)
// elements of a node
static HelmAxes helm_axes(const icarat_ctx *c)
{
  HelmAxes a{};
  const double h[3] = {c->hx, c->hy, c->hz};
  for(int d = 0; d < 3; d++)
  {
    const double md = h[d] / 3.0, mo = h[d] / 6.0, sd = 1.0 / h[d], so = -1.0 / h[d];
    // class 0: only the element above; 1: both; 2: only the element below
    const double m[3][3] = {{0.0, md, mo}, {mo, md + md, mo}, {mo, md, 0.0}};
    const double s[3][3] = {{0.0, sd, so}, {so, sd + sd, so}, {so, sd, 0.0}};
    for(int k = 0; k < 3; k++)
      for(int q = 0; q < 3; q++)
      {
        a.m[d][k][q] = m[k][q];
        a.s[d][k][q] = s[k][q];
      }
  }
  a.c = std::pow(c->helm.radius / (2.0 * std::sqrt(3.0)), 2);
  return a;
}

void helm_free(icarat_ctx *c)
{
  HelmState &H = c->helm;
  if(H.exec)
    cudaGraphExecDestroy(H.exec);
  for(double *p : {H.d_coef, H.d_invd, H.d_F, H.d_val, H.d_r, H.d_z, H.d_p, H.d_Ap,
                   H.d_partials, H.d_oc})
    dfree(p);
  dfree(H.d_cg);
  H = HelmState{};
}

void helm_setup(icarat_ctx *c, double R)
{
  IREQUIRE(R >= 0.0 && std::isfinite(R), ICARAT_ERR_ARG, "filter radius must be >= 0");
  helm_free(c);
  HelmState &H = c->helm;
  H.radius = R;
  helm_element(c->hx, c->hy, c->hz, R, H.ke, H.nj, H.ns);
  double coef[kHelmClasses * 27];
  helm_class_table(H.ke, coef);
  for(int q = 0; q < kHelmClasses; q++)
    H.invd_cls[q] = 1.0 / coef[27 * q + 13];
  const size_t n = (size_t)c->numnp;
  H.d_coef = dalloc(kHelmClasses * 27);
  ICK(cudaMemcpy(H.d_coef, coef, sizeof(coef), cudaMemcpyHostToDevice));
  H.d_invd = dalloc(n);
  H.d_F = dalloc(n);
  H.d_val = dalloc(n);
  H.d_r = dalloc(n);
  H.d_z = dalloc(n);
  H.d_p = dalloc(n);
  H.d_Ap = dalloc(n);
  H.d_partials = dalloc((size_t)kMaxRedBlocks * 2);
  H.d_oc = dalloc(3 * (size_t)c->nelx);
  ICK(cudaMalloc(&H.d_cg, sizeof(CgScalars)));
  ICK(cudaMemsetAsync(H.d_cg, 0, sizeof(CgScalars), c->stream));
  note_launch();
  k_helm_invd<<<blocks_for(n, kHelmThreads, 4 * c->sm_count), kHelmThreads, 0, c->stream>>>(
      hgrid(c), H.d_coef, H.d_invd);
  ICK(cudaGetLastError());
}

// grid of the streaming CG kernels: 8 blocks of 256 threads per SM (full
// occupancy; 4 per SM left them at 3-4 TB/s on the B200)
static int helm_red_blocks(const icarat_ctx *c)
{
  return 8 * c->sm_count < kMaxRedBlocks ? 8 * c->sm_count : kMaxRedBlocks;
}

static void helm_iteration(icarat_ctx *c)
{
  HelmState &H = c->helm;
  const int n = c->numnp;
  const int rb = helm_red_blocks(c);
  const long tiles = (long)((c->NX + kHelmTx - 1) / kHelmTx) *
                    ((c->NY + kHelmTy - 1) / kHelmTy) * ((c->NZ + kHelmTz - 1) / kHelmTz);
  note_launch(3);
  launch_chained(k_helm_spmv, blocks_for(tiles, 1, kMaxRedBlocks), kHelmTx * kHelmWarps, 0,
                 c->stream, hgrid(c), helm_axes(c), H.d_p, H.d_Ap, H.d_partials, H.d_cg);
  HelmInvd iv;
  for(int q = 0; q < kHelmClasses; q++)
    iv.v[q] = H.invd_cls[q];
  (void)n;
  launch_chained(k_helm_update, rb, kRedThreads, 0, c->stream, hgrid(c), iv, H.d_val, H.d_r,
                 H.d_p, H.d_Ap, H.d_partials, H.d_cg);
  launch_chained(k_helm_pupdate, rb, kRedThreads, 0, c->stream, hgrid(c), iv, H.d_r, H.d_p,
                 H.d_cg);
  ICK(cudaGetLastError());
}

// densityFilter (filter_helm.hpp:75-138) of the device vector in (nelx) into
// out (nelx); rtol / maxit of the CG (<= 0: the reference's 1e-10 / 10000)
int helm_filter(icarat_ctx *c, const double *in, double *out, bool is_sens, double rtol,
                int maxit, icarat_solve_info *info)
{
  HelmState &H = c->helm;
  IREQUIRE(H.d_coef != nullptr, ICARAT_ERR_STATE, "Helmholtz filter not set up");
  IREQUIRE(std::isfinite(rtol), ICARAT_ERR_ARG, "rtol must be finite");
  if(rtol <= 0.0)
    rtol = 1.0e-10;
  if(maxit <= 0)
    maxit = 10000;
  const int n = c->numnp;
  const int eb = blocks_for(n, kHelmThreads, 4 * c->sm_count);
  HelmWeights w;
  for(int a = 0; a < 8; a++)
  {
    w.nj[a] = H.nj[a];
    w.ns[a] = H.ns[a];
  }
  note_launch(2);
  k_helm_rhs<<<eb, kHelmThreads, 0, c->stream>>>(hgrid(c), w, in, H.d_F, is_sens ? 1 : 0);
  ICK(cudaGetLastError());
  k_cg_init<<<helm_red_blocks(c), kRedThreads, 0, c->stream>>>(n, H.d_F, H.d_invd, H.d_val,
                                                          H.d_r, H.d_z, H.d_p, H.d_partials,
                                                          H.d_cg, rtol, maxit, 1);
  ICK(cudaGetLastError());
  if(!H.exec)
  {
    cudaGraph_t graph;
    ICK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    set_capturing(true);
    try
    {
      for(int k = 0; k < kHelmChunk; k++)
        helm_iteration(c);
    }
    catch(...)
    {
      set_capturing(false);
      cudaStreamEndCapture(c->stream, &graph);
      throw;
    }
    set_capturing(false);
    ICK(cudaStreamEndCapture(c->stream, &graph));
    ICK(cudaGraphInstantiate(&H.exec, graph, 0));
    cudaGraphDestroy(graph);
  }
  const long max_chunks = ((long)maxit + 1 + kHelmChunk - 1) / kHelmChunk + 1;
  for(long ch = 0; ch < max_chunks; ch++)
  {
    ICK(cudaMemcpyAsync(c->h_cg, H.d_cg, sizeof(CgScalars), cudaMemcpyDeviceToHost,
                        c->stream));
    ICK(cudaStreamSynchronize(c->stream));
    if(c->h_cg->done)
      break;
    ICK(cudaGraphLaunch(H.exec, c->stream));
    note_launch(3 * kHelmChunk);
  }
  note_launch();
  k_helm_out<<<blocks_for(c->nelx, kHelmThreads, 4 * c->sm_count), kHelmThreads, 0,
               c->stream>>>(hgrid(c), w, H.d_val, out, is_sens ? 1 : 0);
  ICK(cudaGetLastError());
  ICK(cudaMemcpyAsync(c->h_cg, H.d_cg, sizeof(CgScalars), cudaMemcpyDeviceToHost,
                      c->stream));
  ICK(cudaStreamSynchronize(c->stream));
  const CgScalars &s = *c->h_cg;
  const int status = s.done ? s.status : ICARAT_WARN_MAXITER;
  if(info)
  {
    *info = icarat_solve_info{};
    info->iterations = s.iter;
    info->rel_residual = s.bnorm > 0 ? s.rnorm / s.bnorm : 0.0;
    info->status = status;
  }
  return status;
}

} // namespace icarat_b200
