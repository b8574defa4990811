// Radius density filter on the voxel grid (Filter<E,N>,
// src/optimization/filter.hpp).
//
// On a MeshIcarat box the neighbour list of preNeighbour (:254-297) is the
// same stencil for every element, clipped at the box faces: offsets (di, dj,
// dk) whose centroid distance d <= R, visited in ascending neighbour element
// id (dk, dj, di lexicographic), weight w = R - d.  The kernels accumulate in
// that order with separate multiply and add (no contraction), so forward and
// transposed results match the reference loop operation for operation.
#include <cmath>

#include "internal.cuh"

namespace icarat_b200
{

// box elements; mask (null without a selection): 1 on the elements a
// selection keeps.  Removed elements are no neighbours and get 0.
struct ElemGrid
{
  int nx, ny, nz, nelx;
  const uint8_t *mask;
};

// dfilters_ds: a_i = sum over valid neighbours of w (geometry only)
__global__ void k_filter_aa(ElemGrid g, int nofs, const int *__restrict__ ofs,
                            const double *__restrict__ w, double *__restrict__ aa)
{
  for(int e = blockIdx.x * blockDim.x + threadIdx.x; e < g.nelx;
      e += gridDim.x * blockDim.x)
  {
    if(g.mask && !g.mask[e])
    {
      aa[e] = 0.0;
      continue;
    }
    const int i = e % g.nx, j = (e / g.nx) % g.ny, k = e / (g.nx * g.ny);
    double a = 0.0;
    for(int q = 0; q < nofs; q++)
    {
      const int ii = i + ofs[3 * q], jj = j + ofs[3 * q + 1], kk = k + ofs[3 * q + 2];
      if(ii < 0 || ii >= g.nx || jj < 0 || jj >= g.ny || kk < 0 || kk >= g.nz)
        continue;
      if(g.mask && !g.mask[ii + (long)jj * g.nx + (long)kk * g.nx * g.ny])
        continue;
      a = __dadd_rn(a, w[q]);
    }
    aa[e] = a;
  }
}

// forward: out_i = sum w x_j / sum w   (filter.hpp:118-137)
__global__ void k_filter_fwd(ElemGrid g, int nofs, const int *__restrict__ ofs,
                             const double *__restrict__ w,
                             const double *__restrict__ in, double *__restrict__ out)
{
  for(int e = blockIdx.x * blockDim.x + threadIdx.x; e < g.nelx;
      e += gridDim.x * blockDim.x)
  {
    if(g.mask && !g.mask[e])
    {
      out[e] = 0.0;
      continue;
    }
    const int i = e % g.nx, j = (e / g.nx) % g.ny, k = e / (g.nx * g.ny);
    double a = 0.0, b = 0.0;
    for(int q = 0; q < nofs; q++)
    {
      const int ii = i + ofs[3 * q], jj = j + ofs[3 * q + 1], kk = k + ofs[3 * q + 2];
      if(ii < 0 || ii >= g.nx || jj < 0 || jj >= g.ny || kk < 0 || kk >= g.nz)
        continue;
      const long f = ii + (long)jj * g.nx + (long)kk * g.nx * g.ny;
      if(g.mask && !g.mask[f])
        continue;
      const double wq = w[q];
      a = __dadd_rn(a, wq);
      b = __dadd_rn(b, __dmul_rn(wq, __ldg(in + f)));
    }
    out[e] = __ddiv_rn(b, a);
  }
}

// n / b rounded to nearest from y = RN(1 / b): q0 = RN(n y) is within one ulp
// of n / b, the remainder n - b q0 is exact in one FMA, and RN(q0 + r y) is
// the correctly rounded quotient (Markstein's theorem: P. Markstein, "Computation
// of elementary functions on the IBM RISC System/6000 processor", IBM J. Res.
// Dev. 34 (1990); Muller et al., Handbook of Floating-Point Arithmetic, on
// division with a fused multiply-add), for normal operands as here (sums of
// positive filter weights, finite terms).  Two FMAs and a product instead of
// a full division per term; the transposed filters stay bit-identical to the
// per-term division of the reference.
__device__ __forceinline__ double div_by_recip(double n, double b, double y)
{
  const double q0 = __dmul_rn(n, y);
  const double r = __fma_rn(-q0, b, n);
  return __fma_rn(r, y, q0);
}

// ra = RN(1 / aa) (IEEE division, once per filter set-up)
__global__ void k_filter_recip(int n, const double *__restrict__ aa, double *__restrict__ ra)
{
  for(int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x)
    ra[e] = __ddiv_rn(1.0, aa[e]);
}

// transposed: out_i = sum_j w_ij in_j / a_j   (filter.hpp:145-152)
__global__ void k_filter_trans(ElemGrid g, int nofs, const int *__restrict__ ofs,
                               const double *__restrict__ w,
                               const double *__restrict__ aa,
                               const double *__restrict__ ra,
                               const double *__restrict__ in,
                               double *__restrict__ out)
{
  for(int e = blockIdx.x * blockDim.x + threadIdx.x; e < g.nelx;
      e += gridDim.x * blockDim.x)
  {
    if(g.mask && !g.mask[e])
    {
      out[e] = 0.0;
      continue;
    }
    const int i = e % g.nx, j = (e / g.nx) % g.ny, k = e / (g.nx * g.ny);
    double s = 0.0;
    for(int q = 0; q < nofs; q++)
    {
      const int ii = i + ofs[3 * q], jj = j + ofs[3 * q + 1], kk = k + ofs[3 * q + 2];
      if(ii < 0 || ii >= g.nx || jj < 0 || jj >= g.ny || kk < 0 || kk >= g.nz)
        continue;
      const long f = ii + (long)jj * g.nx + (long)kk * g.nx * g.ny;
      if(g.mask && !g.mask[f])
        continue;
      s = __dadd_rn(s, div_by_recip(__dmul_rn(w[q], __ldg(in + f)), __ldg(aa + f), __ldg(ra + f)));
    }
    out[e] = s;
  }
}

// the transposed filter of two inputs in one pass (the loop's objective and
// volume sensitivities): neighbour offsets, weights and a_j read once, each
// output summed in the order and with the operations of k_filter_trans
__global__ void k_filter_trans2(ElemGrid g, int nofs, const int *__restrict__ ofs,
                                const double *__restrict__ w, const double *__restrict__ aa,
                                const double *__restrict__ ra,
                                const double *__restrict__ in1, const double *__restrict__ in2,
                                double *__restrict__ out1, double *__restrict__ out2)
{
  for(int e = blockIdx.x * blockDim.x + threadIdx.x; e < g.nelx;
      e += gridDim.x * blockDim.x)
  {
    if(g.mask && !g.mask[e])
    {
      out1[e] = 0.0;
      out2[e] = 0.0;
      continue;
    }
    const int i = e % g.nx, j = (e / g.nx) % g.ny, k = e / (g.nx * g.ny);
    double s1 = 0.0, s2 = 0.0;
    for(int q = 0; q < nofs; q++)
    {
      const int ii = i + ofs[3 * q], jj = j + ofs[3 * q + 1], kk = k + ofs[3 * q + 2];
      if(ii < 0 || ii >= g.nx || jj < 0 || jj >= g.ny || kk < 0 || kk >= g.nz)
        continue;
      const long f = ii + (long)jj * g.nx + (long)kk * g.nx * g.ny;
      if(g.mask && !g.mask[f])
        continue;
      const double wq = w[q], af = __ldg(aa + f), rf = __ldg(ra + f);
      s1 = __dadd_rn(s1, div_by_recip(__dmul_rn(wq, __ldg(in1 + f)), af, rf));
      s2 = __dadd_rn(s2, div_by_recip(__dmul_rn(wq, __ldg(in2 + f)), af, rf));
    }
    out1[e] = s1;
    out2[e] = s2;
  }
}

// sensitivityFilter (filter.hpp:77-104)
__global__ void k_sens_filter(ElemGrid g, int nofs, const int *__restrict__ ofs,
                              const double *__restrict__ w, double vol,
                              const double *__restrict__ s,
                              const double *__restrict__ df, double *__restrict__ out)
{
  for(int e = blockIdx.x * blockDim.x + threadIdx.x; e < g.nelx;
      e += gridDim.x * blockDim.x)
  {
    if(g.mask && !g.mask[e])
    {
      out[e] = 0.0;
      continue;
    }
    const int i = e % g.nx, j = (e / g.nx) % g.ny, k = e / (g.nx * g.ny);
    double a = 0.0, b = 0.0;
    for(int q = 0; q < nofs; q++)
    {
      const int ii = i + ofs[3 * q], jj = j + ofs[3 * q + 1], kk = k + ofs[3 * q + 2];
      if(ii < 0 || ii >= g.nx || jj < 0 || jj >= g.ny || kk < 0 || kk >= g.nz)
        continue;
      const long f = ii + (long)jj * g.nx + (long)kk * g.nx * g.ny;
      if(g.mask && !g.mask[f])
        continue;
      const double wq = w[q], sf = s[f];
      a = __dadd_rn(a, wq);
      b = __dadd_rn(b, __ddiv_rn(__dmul_rn(__dmul_rn(wq, sf), df[f]),
                                 __dmul_rn(sf, vol)));
    }
    const double cc = __ddiv_rn(__dmul_rn(s[e], vol), __dmul_rn(s[e], a));
    out[e] = __dmul_rn(cc, b);
  }
}

// threshold / thresholdDerivative (filter.hpp:217-249)
__global__ void k_threshold(int n, const double *__restrict__ in, double beta,
                            double T, double *__restrict__ out, int derivative)
{
  const double tb = tanh(T * beta);
  for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
      i += gridDim.x * blockDim.x)
  {
    const double t = tanh(beta * (in[i] - T));
    out[i] = derivative ? (0.5 * (beta * (1.0 - t * t))) / tb
                        : 0.5 * (tb + t) / tb;
  }
}

static ElemGrid egrid(const icarat_ctx *c)
{
  return ElemGrid{c->nx, c->ny, c->nz, c->nelx, c->d_emask};
}

static int eblocks(const icarat_ctx *c)
{
  int b = (c->nelx + 255) / 256;
  return b < 1 ? 1 : b;
}

void filter_free(icarat_ctx *c)
{
  dfree(c->filt.d_ofs);
  dfree(c->filt.d_w);
  dfree(c->filt.d_aa);
  dfree(c->filt.d_ra);
  c->filt = FilterState{};
}

void filter_setup(icarat_ctx *c, double R)
{
  IREQUIRE(R >= 0.0 && std::isfinite(R), ICARAT_ERR_ARG, "filter radius must be >= 0");
  filter_free(c);
  FilterState &F = c->filt;
  F.radius = R;
  F.rx = (int)std::ceil(R / c->hx);
  F.ry = (int)std::ceil(R / c->hy);
  F.rz = (int)std::ceil(R / c->hz);
  for(int dk = -F.rz; dk <= F.rz; dk++)
    for(int dj = -F.ry; dj <= F.ry; dj++)
      for(int di = -F.rx; di <= F.rx; di++)
      {
        const double x = di * c->hx, y = dj * c->hy, z = dk * c->hz;
        const double d = std::sqrt(x * x + y * y + z * z);
        if(d <= R)
        {
          F.ofs.push_back(di);
          F.ofs.push_back(dj);
          F.ofs.push_back(dk);
          F.w.push_back(R - d);
        }
      }
  F.nofs = (int)F.w.size();
  ICK(cudaMalloc(&F.d_ofs, sizeof(int) * F.ofs.size()));
  ICK(cudaMemcpy(F.d_ofs, F.ofs.data(), sizeof(int) * F.ofs.size(),
                 cudaMemcpyHostToDevice));
  F.d_w = dalloc(F.w.size());
  ICK(cudaMemcpy(F.d_w, F.w.data(), sizeof(double) * F.w.size(),
                 cudaMemcpyHostToDevice));
  F.d_aa = dalloc(c->nelx);
  note_launch();
  k_filter_aa<<<eblocks(c), 256, 0, c->stream>>>(egrid(c), F.nofs, F.d_ofs, F.d_w,
                                                 F.d_aa);
  F.d_ra = dalloc(c->nelx);
  note_launch();
  k_filter_recip<<<eblocks(c), 256, 0, c->stream>>>(c->nelx, F.d_aa, F.d_ra);
  ICK(cudaGetLastError());
  F.have_forward = false;
}

// The forward pass fails like the reference when a weight sum is below 1e-10
// (filter.hpp:130-134); that can only happen for R < 1e-10.
void filter_apply(icarat_ctx *c, const double *in, double *out, bool is_sens)
{
  FilterState &F = c->filt;
  IREQUIRE(F.d_w != nullptr, ICARAT_ERR_STATE, "filter not set up");
  if(!is_sens)
  {
    IREQUIRE(F.radius >= 1.0e-10, ICARAT_ERR_FILTER,
             "coefficient aa is too small in the density filter");
    note_launch();
    k_filter_fwd<<<eblocks(c), 256, 0, c->stream>>>(egrid(c), F.nofs, F.d_ofs, F.d_w,
                                                    in, out);
    F.have_forward = true;
  }
  else
  {
    IREQUIRE(F.have_forward, ICARAT_ERR_STATE,
             "transposed filter needs a forward call first (filter.hpp:140-153)");
    note_launch();
    k_filter_trans<<<eblocks(c), 256, 0, c->stream>>>(egrid(c), F.nofs, F.d_ofs,
                                                      F.d_w, F.d_aa, F.d_ra, in, out);
  }
  ICK(cudaGetLastError());
}

// transposed filter of in1 and in2 (a forward call must have come first)
void filter_trans2(icarat_ctx *c, const double *in1, const double *in2, double *out1,
                   double *out2)
{
  FilterState &F = c->filt;
  IREQUIRE(F.d_w != nullptr, ICARAT_ERR_STATE, "filter not set up");
  IREQUIRE(F.have_forward, ICARAT_ERR_STATE,
           "transposed filter needs a forward call first (filter.hpp:140-153)");
  note_launch();
  k_filter_trans2<<<eblocks(c), 256, 0, c->stream>>>(egrid(c), F.nofs, F.d_ofs, F.d_w, F.d_aa,
                                                     F.d_ra, in1, in2, out1, out2);
  ICK(cudaGetLastError());
}

void sensitivity_filter_dev(icarat_ctx *c, const double *s, const double *df,
                            double *out)
{
  FilterState &F = c->filt;
  IREQUIRE(F.d_w != nullptr, ICARAT_ERR_STATE, "filter not set up");
  note_launch();
  k_sens_filter<<<eblocks(c), 256, 0, c->stream>>>(egrid(c), F.nofs, F.d_ofs, F.d_w,
                                                   c->vol0, s, df, out);
  ICK(cudaGetLastError());
}

void threshold_dev(icarat_ctx *c, const double *in, double beta, double T,
                   double *out, bool derivative)
{
  note_launch();
  k_threshold<<<eblocks(c), 256, 0, c->stream>>>(c->nelx, in, beta, T, out,
                                                 derivative ? 1 : 0);
  ICK(cudaGetLastError());
}

} // namespace icarat_b200
