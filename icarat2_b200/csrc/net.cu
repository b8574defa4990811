// Learned preconditioner: a 3-D U-net on the node grid (no reference
// counterpart), trained and run by the kernels in this file.
//
// Network (4 levels, 16 base channels; the numpy restatement in
// oracle/net_oracle.py is the checker of these kernels):
//   in(4: residual x/y/z divided by its L2 norm over free DOFs, node density)
//   L0 conv3 4->16 relu, conv3 16->16 relu = S0      pool2
//   L1 conv3 16->32 relu, conv3 32->32 relu = S1     pool2
//   L2 conv3 32->64 relu, conv3 64->64 relu = S2     pool2
//   L3 conv3 64->128 relu, conv3 128->128 relu = B3
//   up2(B3)++S2: conv3 192->64 relu, 64->64 relu = D2
//   up2(D2)++S1: conv3 96->32 relu, 32->32 relu = D1
//   up2(D1)++S0: conv3 48->16 relu, 16->16 relu = D0
//   head conv1 16->3 + bias (FP32): the direction of K^-1 r (training loss
//   1 - cos^2 against the solver's solution, so the scale is left free)
// Storage: activations and weights in BF16 (round to nearest even from the
// FP32 master weights), every sum in FP32, gradients in FP32.  The grid is
// the node grid zero-padded to multiples of 8 (three 2x poolings).
// Layout: tensor [channel][z][y][x] over the padded grid.
//
// Kernels: the forward 3x3x3 convolutions run on the tensor cores
// (k_conv3_tc in net_tc.cu: implicit GEMM, tcgen05, FP32 accumulation in
// TMEM); the backward pass on the CUDA cores (FP32 FMA on BF16 operands):
//   k_conv3        one voxel x 16 output channels per thread, the weights of
//                  a 16-input-channel chunk staged in shared memory: the
//                  data gradient (input: ReLU-masked FP32 output gradient,
//                  weights transposed and flipped)
//   k_conv3_wgrad  per 256-voxel chunk and 16 output channels, every
//                  (input channel, tap) pair summed over the chunk; chunks
//                  reduced in a fixed order (k_chunk_reduce)
//   pooling, nearest upsampling into a channel slice, the 1x1 head, the
//   relative squared error and Adam.
#include <cuda_bf16.h>

#include <cmath>
#include <random>

#include "internal.cuh"

namespace icarat_b200
{
void from_full(icarat_ctx *c, const double *full_in, double *numeq_out, bool host_dst);
void to_full(icarat_ctx *c, const double *numeq_in, double *full_out, bool host_src);

typedef __nv_bfloat16 bf16;

struct NetLayer
{
  int cin, cout, k;
  long woff, boff; // offsets of W[cout][cin][k^3] and b[cout] in the flat vector
};

static const int kLayers[15][3] = {{4, 16, 3},   {16, 16, 3}, {16, 32, 3},  {32, 32, 3},
                                   {32, 64, 3},  {64, 64, 3}, {64, 128, 3}, {128, 128, 3},
                                   {192, 64, 3}, {64, 64, 3}, {96, 32, 3},  {32, 32, 3},
                                   {48, 16, 3},  {16, 16, 3}, {16, 3, 1}};

// ---------------------------------------------------------------- kernels
struct Dims
{
  int X, Y, Z; // padded extents of this level
  long V;      // voxels
};

__device__ __forceinline__ float bfv(bf16 v) { return __bfloat162float(v); }

// y[co][v] (co in [16 blockIdx.y, +16)) = sum_ci sum_tap W[co][ci][tap] x[ci][v + tap]
// (+ bias, relu, BF16 out) or plain FP32 out.  MASK: the input is an FP32
// gradient taken where the (BF16) tensor xmask > 0.
template <typename TI, bool MASK, bool OUT_BF16>
__global__ void __launch_bounds__(128)
    k_conv3(Dims d, const TI *__restrict__ x, const bf16 *__restrict__ xmask, int cin,
            const bf16 *__restrict__ W, const float *__restrict__ bias, int cout,
            bf16 *__restrict__ yb, float *__restrict__ yf, int relu)
{
  __shared__ float Ws[16][27][16]; // [ci in chunk][tap][co in tile]
  const int co0 = blockIdx.y * 16;
  const long v = blockIdx.x * (long)blockDim.x + threadIdx.x;
  const bool valid = v < d.V;
  const int vx = valid ? (int)(v % d.X) : 0;
  const int vy = valid ? (int)((v / d.X) % d.Y) : 0;
  const int vz = valid ? (int)(v / ((long)d.X * d.Y)) : 0;
  unsigned inb = 0; // bit tap: neighbour inside the grid
#pragma unroll
  for(int tap = 0; tap < 27; tap++)
  {
    const int xx = vx + tap % 3 - 1, yy = vy + (tap / 3) % 3 - 1, zz = vz + tap / 9 - 1;
    if(valid && xx >= 0 && xx < d.X && yy >= 0 && yy < d.Y && zz >= 0 && zz < d.Z)
      inb |= 1u << tap;
  }
  float acc[16];
#pragma unroll
  for(int q = 0; q < 16; q++)
    acc[q] = 0.0f;
  for(int ci0 = 0; ci0 < cin; ci0 += 16)
  {
    const int nc = min(16, cin - ci0);
    __syncthreads();
    for(int q = threadIdx.x; q < 16 * 27 * 16; q += blockDim.x)
    {
      const int co = q % 16, tap = (q / 16) % 27, ci = q / (16 * 27);
      Ws[ci][tap][co] = (ci < nc && co0 + co < cout)
                            ? bfv(W[((long)(co0 + co) * cin + ci0 + ci) * 27 + tap])
                            : 0.0f;
    }
    __syncthreads();
    for(int ci = 0; ci < nc; ci++)
    {
      const TI *xc = x + (long)(ci0 + ci) * d.V;
      const bf16 *mc = MASK ? xmask + (long)(ci0 + ci) * d.V : nullptr;
#pragma unroll
      for(int tap = 0; tap < 27; tap++)
      {
        if(!((inb >> tap) & 1u))
          continue;
        const long off = v + (tap % 3 - 1) + (long)((tap / 3) % 3 - 1) * d.X +
                         (long)(tap / 9 - 1) * d.X * d.Y;
        float xv;
        if constexpr(MASK)
          xv = bfv(mc[off]) > 0.0f ? (float)xc[off] : 0.0f;
        else
          xv = (float)xc[off];
#pragma unroll
        for(int q = 0; q < 16; q++)
          acc[q] = fmaf(xv, Ws[ci][tap][q], acc[q]);
      }
    }
  }
  if(!valid)
    return;
#pragma unroll
  for(int q = 0; q < 16; q++)
  {
    const int co = co0 + q;
    if(co >= cout)
      break;
    float y = acc[q] + (bias ? bias[co] : 0.0f);
    if(relu)
      y = fmaxf(y, 0.0f);
    if constexpr(OUT_BF16)
      yb[(long)co * d.V + v] = __float2bfloat16_rn(y);
    else
      yf[(long)co * d.V + v] = y;
  }
}

__device__ __forceinline__ float load_bf_or_f(const bf16 *p) { return bfv(*p); }
__device__ __forceinline__ float load_bf_or_f(const float *p) { return *p; }

// part[chunk][co][ci][tap] = sum over the chunk's voxels of dy[co][v] x[ci][v+tap],
// dy taken where ymask > 0.
__global__ void __launch_bounds__(128)
    k_conv3_wgrad(Dims d, const bf16 *__restrict__ x, int cin, const float *__restrict__ dy,
                  const bf16 *__restrict__ ymask, int cout, float *__restrict__ part)
{
  constexpr int CH = 256;
  __shared__ float dys[16][CH];
  __shared__ int vxyz[CH][3]; // coordinates of the chunk's voxels (one division each)
  const int chunk = blockIdx.x, co0 = blockIdx.y * 16;
  const long v0 = (long)chunk * CH;
  for(int i = threadIdx.x; i < CH; i += blockDim.x)
  {
    const long v = v0 + i;
    const int vx = (int)(v % d.X);
    const long r = v / d.X;
    vxyz[i][0] = vx;
    vxyz[i][1] = (int)(r % d.Y);
    vxyz[i][2] = (int)(r / d.Y);
  }
  for(int q = threadIdx.x; q < 16 * CH; q += blockDim.x)
  {
    const int co = q / CH, i = q % CH;
    const long v = v0 + i;
    float g = 0.0f;
    if(v < d.V && co0 + co < cout)
    {
      const long id = (long)(co0 + co) * d.V + v;
      g = bfv(ymask[id]) > 0.0f ? dy[id] : 0.0f;
    }
    dys[co][i] = g;
  }
  __syncthreads();
  const int npair = cin * 27;
  for(int p = threadIdx.x; p < npair; p += blockDim.x)
  {
    const int ci = p / 27, tap = p % 27;
    const int ox = tap % 3 - 1, oy = (tap / 3) % 3 - 1, oz = tap / 9 - 1;
    const bf16 *xc = x + (long)ci * d.V;
    float acc[16];
#pragma unroll
    for(int q = 0; q < 16; q++)
      acc[q] = 0.0f;
    for(int i = 0; i < CH; i++)
    {
      const long v = v0 + i;
      if(v >= d.V)
        break;
      const int xx = vxyz[i][0] + ox, yy = vxyz[i][1] + oy, zz = vxyz[i][2] + oz;
      if(xx < 0 || xx >= d.X || yy < 0 || yy >= d.Y || zz < 0 || zz >= d.Z)
        continue;
      const float xv = bfv(xc[v + ox + (long)oy * d.X + (long)oz * d.X * d.Y]);
#pragma unroll
      for(int q = 0; q < 16; q++)
        acc[q] = fmaf(xv, dys[q][i], acc[q]);
    }
#pragma unroll
    for(int q = 0; q < 16; q++)
      if(co0 + q < cout)
        part[((long)chunk * cout + co0 + q) * npair + p] = acc[q];
  }
}

// g[i] = sum_chunk part[chunk][i] (fixed order)
__global__ void k_chunk_reduce(long n, int nchunks, const float *__restrict__ part,
                               float *__restrict__ g)
{
  for(long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
      i += (long)gridDim.x * blockDim.x)
  {
    float s = 0.0f;
    for(int c = 0; c < nchunks; c++)
      s += part[(long)c * n + i];
    g[i] = s;
  }
}

// db[co] = sum_v dy[co][v] where ymask > 0 (ymask null: everywhere)
__global__ void k_bias_grad(Dims d, const float *__restrict__ dy, const bf16 *__restrict__ ymask,
                            float *__restrict__ db)
{
  __shared__ double sh[32];
  const int co = blockIdx.x;
  double s = 0.0;
  for(long v = threadIdx.x; v < d.V; v += blockDim.x)
  {
    const long id = (long)co * d.V + v;
    if(!ymask || bfv(ymask[id]) > 0.0f)
      s += dy[id];
  }
  double a[1] = {s};
  block_sum<1>(a, sh);
  if(threadIdx.x == 0)
    db[co] = (float)a[0];
}

// The grid transfers run one block per x-line (channel, z, y) of the grid
// they write, threads along x: no 64-bit index division per element.
// Blocks for the x-lines of ch channels of level d.
static inline int line_blocks(int ch, int Z, int Y) { return std::min(ch * Z * Y, 148 * 16); }

// coarse[c][V] = mean of the 8 children
__global__ void k_pool(Dims f, Dims c, int ch, const bf16 *__restrict__ in, bf16 *__restrict__ out)
{
  const int lines = ch * c.Z * c.Y;
  for(int L = blockIdx.x; L < lines; L += gridDim.x)
  {
    const int Y = L % c.Y, Z = (L / c.Y) % c.Z, k = L / (c.Y * c.Z);
    const bf16 *src = in + (long)k * f.V + (long)(2 * Z) * f.X * f.Y + (long)(2 * Y) * f.X;
    bf16 *dst = out + (long)k * c.V + (long)Z * c.X * c.Y + (long)Y * c.X;
    for(int X = threadIdx.x; X < c.X; X += blockDim.x)
    {
      float s = 0.0f;
      for(int q = 0; q < 8; q++)
        s += bfv(src[(2 * X + (q & 1)) + (long)((q >> 1) & 1) * f.X +
                     (long)(q >> 2) * f.X * f.Y]);
      dst[X] = __float2bfloat16_rn(s * 0.125f);
    }
  }
}

// fine[c][v] += coarse gradient / 8 (the pooling's adjoint)
__global__ void k_pool_back_add(Dims f, Dims c, int ch, const float *__restrict__ dc,
                                float *__restrict__ df)
{
  const int lines = ch * f.Z * f.Y;
  for(int L = blockIdx.x; L < lines; L += gridDim.x)
  {
    const int y = L % f.Y, z = (L / f.Y) % f.Z, k = L / (f.Y * f.Z);
    const float *src = dc + (long)k * c.V + (long)(z / 2) * c.X * c.Y + (long)(y / 2) * c.X;
    float *dst = df + (long)k * f.V + (long)z * f.X * f.Y + (long)y * f.X;
    for(int x = threadIdx.x; x < f.X; x += blockDim.x)
      dst[x] += 0.125f * src[x / 2];
  }
}

// fine[c][v] = coarse (nearest)
__global__ void k_up(Dims f, Dims c, int ch, const bf16 *__restrict__ in, bf16 *__restrict__ out)
{
  const int lines = ch * f.Z * f.Y;
  for(int L = blockIdx.x; L < lines; L += gridDim.x)
  {
    const int y = L % f.Y, z = (L / f.Y) % f.Z, k = L / (f.Y * f.Z);
    const bf16 *src = in + (long)k * c.V + (long)(z / 2) * c.X * c.Y + (long)(y / 2) * c.X;
    bf16 *dst = out + (long)k * f.V + (long)z * f.X * f.Y + (long)y * f.X;
    if(f.X % 8 == 0 && c.X % 4 == 0)
    {
      // 8 outputs from 4 inputs per thread: 16-byte stores, 8-byte loads
      // (every line starts on those boundaries when the extents divide)
      for(int x = 8 * threadIdx.x; x < f.X; x += 8 * blockDim.x)
      {
        const uint2 s4 = *reinterpret_cast<const uint2 *>(src + x / 2);
        const uint32_t a = s4.x & 0xFFFFu, b = s4.x >> 16, cc = s4.y & 0xFFFFu, dd = s4.y >> 16;
        *reinterpret_cast<uint4 *>(dst + x) =
            make_uint4(a | (a << 16), b | (b << 16), cc | (cc << 16), dd | (dd << 16));
      }
    }
    else
      for(int x = threadIdx.x; x < f.X; x += blockDim.x)
        dst[x] = src[x / 2];
  }
}

// coarse gradient = sum of the 8 children (the upsampling's adjoint)
__global__ void k_up_back(Dims f, Dims c, int ch, const float *__restrict__ df,
                          float *__restrict__ dc)
{
  const int lines = ch * c.Z * c.Y;
  for(int L = blockIdx.x; L < lines; L += gridDim.x)
  {
    const int Y = L % c.Y, Z = (L / c.Y) % c.Z, k = L / (c.Y * c.Z);
    const float *src = df + (long)k * f.V + (long)(2 * Z) * f.X * f.Y + (long)(2 * Y) * f.X;
    float *dst = dc + (long)k * c.V + (long)Z * c.X * c.Y + (long)Y * c.X;
    for(int X = threadIdx.x; X < c.X; X += blockDim.x)
    {
      float s = 0.0f;
      for(int q = 0; q < 8; q++)
        s += src[(2 * X + (q & 1)) + (long)((q >> 1) & 1) * f.X + (long)(q >> 2) * f.X * f.Y];
      dst[X] = s;
    }
  }
}

// head: out[c][v] = b[c] + sum_ci W[c][ci] x[ci][v]  (FP32)
__global__ void k_head(Dims d, const bf16 *__restrict__ x, const bf16 *__restrict__ W,
                       const float *__restrict__ b, float *__restrict__ out)
{
  for(long v = blockIdx.x * (long)blockDim.x + threadIdx.x; v < d.V;
      v += (long)gridDim.x * blockDim.x)
  {
    float xv[16];
#pragma unroll
    for(int ci = 0; ci < 16; ci++)
      xv[ci] = bfv(x[(long)ci * d.V + v]);
#pragma unroll
    for(int c = 0; c < 3; c++)
    {
      float s = b[c];
#pragma unroll
      for(int ci = 0; ci < 16; ci++)
        s = fmaf(bfv(W[c * 16 + ci]), xv[ci], s);
      out[(long)c * d.V + v] = s;
    }
  }
}

// head backward: dx[ci][v] = sum_c W[c][ci] dout[c][v]
__global__ void k_head_back(Dims d, const float *__restrict__ dout, const bf16 *__restrict__ W,
                            float *__restrict__ dx)
{
  for(long v = blockIdx.x * (long)blockDim.x + threadIdx.x; v < d.V;
      v += (long)gridDim.x * blockDim.x)
  {
    const float g0 = dout[v], g1 = dout[d.V + v], g2 = dout[2 * d.V + v];
#pragma unroll
    for(int ci = 0; ci < 16; ci++)
      dx[(long)ci * d.V + v] =
          bfv(W[ci]) * g0 + bfv(W[16 + ci]) * g1 + bfv(W[32 + ci]) * g2;
  }
}

// dW[c][ci] = sum_v dout[c][v] x[ci][v]: one block per (c, ci)
__global__ void k_head_wgrad(Dims d, const float *__restrict__ dout, const bf16 *__restrict__ x,
                             float *__restrict__ dW)
{
  __shared__ double sh[32];
  const int c = blockIdx.x / 16, ci = blockIdx.x % 16;
  double s = 0.0;
  for(long v = threadIdx.x; v < d.V; v += blockDim.x)
    s += (double)dout[(long)c * d.V + v] * (double)bfv(x[(long)ci * d.V + v]);
  double a[1] = {s};
  block_sum<1>(a, sh);
  if(threadIdx.x == 0)
    dW[c * 16 + ci] = (float)a[0];
}

// Network input from a node vector (component-major, FP64 or FP32) scaled by
// 1 / s, and the node density from the element densities; zero padding.
template <typename T>
__global__ void k_net_input(Dims d, GridDev g, const T *__restrict__ r, const uint8_t *__restrict__ fix,
                            const double *__restrict__ rho, float inv_s, bf16 *__restrict__ in)
{
  for(long v = blockIdx.x * (long)blockDim.x + threadIdx.x; v < d.V;
      v += (long)gridDim.x * blockDim.x)
  {
    const int x = (int)(v % d.X), y = (int)((v / d.X) % d.Y), z = (int)(v / ((long)d.X * d.Y));
    float ch[4] = {0.f, 0.f, 0.f, 0.f};
    if(x < g.NX && y < g.NY && z < g.NZ)
    {
      const long n = x + (long)y * g.NX + (long)z * g.NX * g.NY;
      const unsigned f = fix[n];
#pragma unroll
      for(int c = 0; c < 3; c++)
        ch[c] = ((f >> c) & 1u) ? 0.0f : (float)r[(long)c * g.numnp + n] * inv_s;
      double s = 0.0;
      int cnt = 0;
      for(int q = 0; q < 8; q++)
      {
        const int ex = x - 1 + (q & 1), ey = y - 1 + ((q >> 1) & 1), ez = z - 1 + (q >> 2);
        if(ex >= 0 && ex < g.nx && ey >= 0 && ey < g.ny && ez >= 0 && ez < g.nz)
        {
          s += rho[ex + (long)ey * g.nx + (long)ez * g.nx * g.ny];
          cnt++;
        }
      }
      ch[3] = cnt ? (float)(s / cnt) : 0.0f;
    }
#pragma unroll
    for(int c = 0; c < 4; c++)
      in[(long)c * d.V + v] = __float2bfloat16_rn(ch[c]);
  }
}

// Net output [3][V] -> node vector s * out (constrained components 0)
template <typename T>
__global__ void k_net_output(Dims d, GridDev g, const float *__restrict__ out,
                             const uint8_t *__restrict__ fix, double s, T *__restrict__ z)
{
  for(long n = blockIdx.x * (long)blockDim.x + threadIdx.x; n < g.numnp;
      n += (long)gridDim.x * blockDim.x)
  {
    const int x = (int)(n % g.NX), y = (int)((n / g.NX) % g.NY), zz = (int)(n / ((long)g.NX * g.NY));
    const long v = x + (long)y * d.X + (long)zz * d.X * d.Y;
    const unsigned f = fix[n];
#pragma unroll
    for(int c = 0; c < 3; c++)
      z[(long)c * g.numnp + n] = ((f >> c) & 1u) ? T(0) : (T)(s * out[(long)c * d.V + v]);
  }
}

// Target t = u / s on the padded grid (0 outside / constrained), with the
// mask of counted entries, and partial sums of t^2.
__global__ void k_net_target(Dims d, GridDev g, const double *__restrict__ u,
                             const uint8_t *__restrict__ fix, double inv_s, float *__restrict__ t,
                             uint8_t *__restrict__ m)
{
  for(long v = blockIdx.x * (long)blockDim.x + threadIdx.x; v < d.V;
      v += (long)gridDim.x * blockDim.x)
  {
    const int x = (int)(v % d.X), y = (int)((v / d.X) % d.Y), z = (int)(v / ((long)d.X * d.Y));
    const bool in = x < g.NX && y < g.NY && z < g.NZ;
    const long n = in ? x + (long)y * g.NX + (long)z * g.NX * g.NY : 0;
    const unsigned f = in ? fix[n] : 7u;
#pragma unroll
    for(int c = 0; c < 3; c++)
    {
      const bool use = !((f >> c) & 1u);
      t[(long)c * d.V + v] = use ? (float)(u[(long)c * g.numnp + n] * inv_s) : 0.0f;
      m[(long)c * d.V + v] = use ? 1 : 0;
    }
  }
}

// loss partials over the mask (FP64): y . t, y . y, t . t
__global__ void k_net_loss(long n, const float *__restrict__ out, const float *__restrict__ t,
                           const uint8_t *__restrict__ m, double *__restrict__ partials)
{
  __shared__ double sh[96];
  double yt = 0.0, yy = 0.0, tt = 0.0;
  for(long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
      i += (long)gridDim.x * blockDim.x)
    if(m[i])
    {
      const double y = out[i], ti = t[i];
      yt += y * ti;
      yy += y * y;
      tt += ti * ti;
    }
  double a[3] = {yt, yy, tt};
  block_sum<3>(a, sh);
  if(threadIdx.x == 0)
  {
    partials[3 * blockIdx.x] = a[0];
    partials[3 * blockIdx.x + 1] = a[1];
    partials[3 * blockIdx.x + 2] = a[2];
  }
}

constexpr double kNetNormPenalty = 1e-2;

// dL/dy of L = 1 - (y.t)^2 / (|y|^2 |t|^2) + mu (|y|^2 - 1)^2: ct t + cy y
// on the mask
__global__ void k_net_dout(long n, const float *__restrict__ out, const float *__restrict__ t,
                           const uint8_t *__restrict__ m, float ct, float cy,
                           float *__restrict__ dout)
{
  for(long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
      i += (long)gridDim.x * blockDim.x)
    dout[i] = m[i] ? ct * t[i] + cy * out[i] : 0.0f;
}

struct LayerTable
{
  int cin[15], cout[15], k[15];
  long woff[15], boff[15];
};

// BF16 copies of the weights: wb[i] = w[i]; wt = per layer W^T with flipped taps
__global__ void k_net_weights(long n, LayerTable lt, const float *__restrict__ w,
                              bf16 *__restrict__ wb, bf16 *__restrict__ wt)
{
  for(long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
      i += (long)gridDim.x * blockDim.x)
  {
    const bf16 h = __float2bfloat16_rn(w[i]);
    wb[i] = h;
    for(int l = 0; l < 15; l++)
    {
      const long nw = (long)lt.cout[l] * lt.cin[l] * lt.k[l] * lt.k[l] * lt.k[l];
      if(i >= lt.woff[l] && i < lt.woff[l] + nw)
      {
        const int kk = lt.k[l] * lt.k[l] * lt.k[l];
        const long j = i - lt.woff[l];
        const int tap = (int)(j % kk), ci = (int)((j / kk) % lt.cin[l]), co = (int)(j / kk / lt.cin[l]);
        wt[lt.woff[l] + ((long)ci * lt.cout[l] + co) * kk + (kk - 1 - tap)] = h;
      }
    }
  }
}

__global__ void k_adam(long n, float *__restrict__ w, float *__restrict__ m, float *__restrict__ v,
                       const float *__restrict__ g, float lr, float b1, float b2, float c1,
                       float c2, float eps)
{
  for(long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
      i += (long)gridDim.x * blockDim.x)
  {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  }
}

} // namespace icarat_b200

using namespace icarat_b200;

struct icarat_net
{
  int device = 0;
  NetLayer L[15];
  LayerTable lt;
  long np = 0;
  float *w = nullptr, *m = nullptr, *v = nullptr, *g = nullptr;
  bf16 *wb = nullptr, *wt = nullptr;
  // conv3 weights packed for the tensor-core forward (net_tc.cu) and its
  // error flag (an mbarrier wait that ran out)
  bf16 *wpk = nullptr;
  long wpk_off[15] = {};
  int *tc_err = nullptr;
  long step = 0;
  bool wdirty = true;
  // activations of the current padded grid
  int PX = 0, PY = 0, PZ = 0;
  Dims d[4];
  bf16 *in = nullptr, *a0 = nullptr, *c0 = nullptr, *e0 = nullptr, *d0 = nullptr;
  bf16 *p1 = nullptr, *a1 = nullptr, *c1 = nullptr, *e1 = nullptr, *d1 = nullptr;
  bf16 *p2 = nullptr, *a2 = nullptr, *c2 = nullptr, *e2 = nullptr, *d2 = nullptr;
  bf16 *p3 = nullptr, *a3 = nullptr, *b3 = nullptr;
  float *out = nullptr, *tgt = nullptr, *dout = nullptr;
  uint8_t *mask = nullptr;
  float *gA[4] = {}, *gB[4] = {}, *part = nullptr;
  long part_n = 0;
  double *lpart = nullptr, *h_lpart = nullptr;
  std::vector<void *> act;
};

namespace
{
int nb(long n, int t = 256)
{
  long b = (n + t - 1) / t;
  return (int)std::max(1L, std::min(b, 148L * 32));
}

template <typename T> T *alloc_n(long n)
{
  void *p = nullptr;
  cudaError_t e = cudaMalloc(&p, sizeof(T) * (size_t)std::max(1L, n));
  if(e != cudaSuccess)
    throw Error{ICARAT_ERR_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e)};
  return static_cast<T *>(p);
}

void free_acts(icarat_net *N)
{
  for(void *p : N->act)
    cudaFree(p);
  N->act.clear();
  N->PX = N->PY = N->PZ = 0;
}

// activation and gradient buffers for the padded grid of ctx
void ensure_grid(icarat_net *N, const icarat_ctx *c)
{
  const int PX = (c->NX + 7) / 8 * 8, PY = (c->NY + 7) / 8 * 8, PZ = (c->NZ + 7) / 8 * 8;
  if(PX == N->PX && PY == N->PY && PZ == N->PZ)
    return;
  free_acts(N);
  for(int l = 0; l < 4; l++)
    N->d[l] = Dims{PX >> l, PY >> l, PZ >> l, (long)(PX >> l) * (PY >> l) * (PZ >> l)};
  auto B = [&](long n) {
    bf16 *p = alloc_n<bf16>(n);
    N->act.push_back(p);
    return p;
  };
  auto F = [&](long n) {
    float *p = alloc_n<float>(n);
    N->act.push_back(p);
    return p;
  };
  const long V0 = N->d[0].V, V1 = N->d[1].V, V2 = N->d[2].V, V3 = N->d[3].V;
  N->in = B(4 * V0);
  N->a0 = B(16 * V0);
  N->c0 = B(48 * V0);
  N->e0 = B(16 * V0);
  N->d0 = B(16 * V0);
  N->p1 = B(16 * V1);
  N->a1 = B(32 * V1);
  N->c1 = B(96 * V1);
  N->e1 = B(32 * V1);
  N->d1 = B(32 * V1);
  N->p2 = B(32 * V2);
  N->a2 = B(64 * V2);
  N->c2 = B(192 * V2);
  N->e2 = B(64 * V2);
  N->d2 = B(64 * V2);
  N->p3 = B(64 * V3);
  N->a3 = B(128 * V3);
  N->b3 = B(128 * V3);
  N->out = F(3 * V0);
  N->tgt = F(3 * V0);
  N->dout = F(3 * V0);
  N->mask = (uint8_t *)B((3 * V0 + 1) / 2);
  const int maxc[4] = {48, 96, 192, 128};
  for(int l = 0; l < 4; l++)
  {
    N->gA[l] = F((long)maxc[l] * N->d[l].V);
    N->gB[l] = F((long)maxc[l] * N->d[l].V);
  }
  // weight-gradient partials: the largest chunks x parameters of any layer
  long pn = 0;
  const int lev[15] = {0, 0, 1, 1, 2, 2, 3, 3, 2, 2, 1, 1, 0, 0, 0};
  for(int l = 0; l < 14; l++)
  {
    const long chunks = (N->d[lev[l]].V + 255) / 256;
    pn = std::max(pn, chunks * (long)N->L[l].cin * N->L[l].cout * 27);
  }
  N->part = F(pn);
  N->part_n = pn;
  N->lpart = (double *)F(3 * 4096 * 2);
  N->PX = PX;
  N->PY = PY;
  N->PZ = PZ;
}

void refresh_weights(icarat_net *N, cudaStream_t st)
{
  if(!N->wdirty)
    return;
  note_launch();
  k_net_weights<<<nb(N->np), 256, 0, st>>>(N->np, N->lt, N->w, N->wb, N->wt);
  ICK(cudaGetLastError());
  for(int l = 0; l < 15; l++)
    if(N->L[l].k == 3)
      conv3_tc_pack(reinterpret_cast<const uint16_t *>(N->wb + N->L[l].woff), N->L[l].cin,
                    N->L[l].cout, reinterpret_cast<uint16_t *>(N->wpk + N->wpk_off[l]), st);
  N->wdirty = false;
}

// the tensor-core convolution reports a wait that ran out through a flag
void check_tc_conv(icarat_net *N, cudaStream_t st)
{
  int e = 0;
  ICK(cudaMemcpyAsync(&e, N->tc_err, sizeof(int), cudaMemcpyDeviceToHost, st));
  ICK(cudaStreamSynchronize(st));
  if(e)
  {
    ICK(cudaMemsetAsync(N->tc_err, 0, sizeof(int), st));
    throw Error{ICARAT_ERR_CUDA, "tensor-core convolution: an mbarrier wait ran out"};
  }
}

// forward conv3 + bias + ReLU on the tensor cores (net_tc.cu)
void conv_fwd(icarat_net *N, cudaStream_t st, int li, int lvl, const bf16 *x, bf16 *y)
{
  const NetLayer &Ly = N->L[li];
  const Dims &d = N->d[lvl];
  conv3_tc_fwd(d.X, d.Y, d.Z, d.V, reinterpret_cast<const uint16_t *>(x), Ly.cin,
               reinterpret_cast<const uint16_t *>(N->wpk + N->wpk_off[li]), N->w + Ly.boff,
               Ly.cout, reinterpret_cast<uint16_t *>(y), N->tc_err, st);
}

void forward(icarat_net *N, cudaStream_t st)
{
  const Dims *d = N->d;
  const long V0 = d[0].V, V1 = d[1].V, V2 = d[2].V;
  conv_fwd(N, st, 0, 0, N->in, N->a0);
  conv_fwd(N, st, 1, 0, N->a0, N->c0 + 32 * V0); // S0 into the skip slice
  note_launch(3);
  k_pool<<<line_blocks(16, d[1].Z, d[1].Y), 128, 0, st>>>(d[0], d[1], 16, N->c0 + 32 * V0, N->p1);
  conv_fwd(N, st, 2, 1, N->p1, N->a1);
  conv_fwd(N, st, 3, 1, N->a1, N->c1 + 64 * V1);
  k_pool<<<line_blocks(32, d[2].Z, d[2].Y), 128, 0, st>>>(d[1], d[2], 32, N->c1 + 64 * V1, N->p2);
  conv_fwd(N, st, 4, 2, N->p2, N->a2);
  conv_fwd(N, st, 5, 2, N->a2, N->c2 + 128 * V2);
  k_pool<<<line_blocks(64, d[3].Z, d[3].Y), 128, 0, st>>>(d[2], d[3], 64, N->c2 + 128 * V2, N->p3);
  conv_fwd(N, st, 6, 3, N->p3, N->a3);
  conv_fwd(N, st, 7, 3, N->a3, N->b3);
  note_launch();
  k_up<<<line_blocks(128, d[2].Z, d[2].Y), 128, 0, st>>>(d[2], d[3], 128, N->b3, N->c2);
  conv_fwd(N, st, 8, 2, N->c2, N->e2);
  conv_fwd(N, st, 9, 2, N->e2, N->d2);
  note_launch();
  k_up<<<line_blocks(64, d[1].Z, d[1].Y), 128, 0, st>>>(d[1], d[2], 64, N->d2, N->c1);
  conv_fwd(N, st, 10, 1, N->c1, N->e1);
  conv_fwd(N, st, 11, 1, N->e1, N->d1);
  note_launch();
  k_up<<<line_blocks(32, d[0].Z, d[0].Y), 128, 0, st>>>(d[0], d[1], 32, N->d1, N->c0);
  conv_fwd(N, st, 12, 0, N->c0, N->e0);
  conv_fwd(N, st, 13, 0, N->e0, N->d0);
  note_launch();
  k_head<<<nb(V0), 256, 0, st>>>(d[0], N->d0, N->wb + N->L[14].woff, N->w + N->L[14].boff,
                                 N->out);
  ICK(cudaGetLastError());
}

// Backward of conv layer li (input x at level lvl, output y): dy (FP32, the
// gradient after the ReLU) -> weight and bias gradients, and dx if wanted.
void conv_back(icarat_net *N, cudaStream_t st, int li, int lvl, const bf16 *x, const bf16 *y,
               const float *dy, float *dx)
{
  const NetLayer &Ly = N->L[li];
  const Dims &d = N->d[lvl];
  const int chunks = (int)((d.V + 255) / 256);
  note_launch(3);
  k_conv3_wgrad<<<dim3(chunks, (Ly.cout + 15) / 16), 128, 0, st>>>(d, x, Ly.cin, dy, y, Ly.cout,
                                                                     N->part);
  const long nw = (long)Ly.cout * Ly.cin * 27;
  k_chunk_reduce<<<nb(nw), 256, 0, st>>>(nw, chunks, N->part, N->g + Ly.woff);
  k_bias_grad<<<Ly.cout, 256, 0, st>>>(d, dy, y, N->g + Ly.boff);
  if(dx)
  {
    // dx[ci] = sum_co sum_tap W[co][ci][tap] dy_masked[co][v - tap]
    dim3 grid((unsigned)((d.V + 127) / 128), (unsigned)((Ly.cin + 15) / 16));
    note_launch();
    k_conv3<float, true, false><<<grid, 128, 0, st>>>(d, dy, y, Ly.cout, N->wt + Ly.woff,
                                                      nullptr, Ly.cin, nullptr, dx, 0);
  }
  ICK(cudaGetLastError());
}

void backward(icarat_net *N, cudaStream_t st)
{
  const Dims *d = N->d;
  const long V0 = d[0].V, V1 = d[1].V, V2 = d[2].V;
  // head
  note_launch(3);
  k_head_wgrad<<<48, 256, 0, st>>>(d[0], N->dout, N->d0, N->g + N->L[14].woff);
  k_bias_grad<<<3, 256, 0, st>>>(d[0], N->dout, nullptr, N->g + N->L[14].boff);
  k_head_back<<<nb(V0), 256, 0, st>>>(d[0], N->dout, N->wb + N->L[14].woff, N->gA[0]);
  // level 0 decoder: gA[0] = dD0 -> gB[0] = dE0 -> gA[0] = dC0 (48 ch)
  conv_back(N, st, 13, 0, N->e0, N->d0, N->gA[0], N->gB[0]);
  conv_back(N, st, 12, 0, N->c0, N->e0, N->gB[0], N->gA[0]);
  // dD1 = up^T(dC0[0:32]) -> gA[1]; dS0 (skip) stays in gA[0] + 32 V0
  note_launch();
  k_up_back<<<line_blocks(32, d[1].Z, d[1].Y), 128, 0, st>>>(d[0], d[1], 32, N->gA[0], N->gA[1]);
  conv_back(N, st, 11, 1, N->e1, N->d1, N->gA[1], N->gB[1]);
  conv_back(N, st, 10, 1, N->c1, N->e1, N->gB[1], N->gA[1]); // dC1 (96 ch)
  note_launch();
  k_up_back<<<line_blocks(64, d[2].Z, d[2].Y), 128, 0, st>>>(d[1], d[2], 64, N->gA[1], N->gA[2]);
  conv_back(N, st, 9, 2, N->e2, N->d2, N->gA[2], N->gB[2]);
  conv_back(N, st, 8, 2, N->c2, N->e2, N->gB[2], N->gA[2]); // dC2 (192 ch)
  note_launch();
  k_up_back<<<line_blocks(128, d[3].Z, d[3].Y), 128, 0, st>>>(d[2], d[3], 128, N->gA[2], N->gA[3]);
  // bottom: dB3 = gA[3] -> dA3 = gB[3] -> dP3 = gA[3]
  conv_back(N, st, 7, 3, N->a3, N->b3, N->gA[3], N->gB[3]);
  conv_back(N, st, 6, 3, N->p3, N->a3, N->gB[3], N->gA[3]);
  // dS2 = dC2[128:192] + pool^T(dP3)
  float *dS2 = N->gA[2] + 128 * V2;
  note_launch();
  k_pool_back_add<<<line_blocks(64, d[2].Z, d[2].Y), 128, 0, st>>>(d[2], d[3], 64, N->gA[3], dS2);
  conv_back(N, st, 5, 2, N->a2, N->c2 + 128 * V2, dS2, N->gB[2]);
  conv_back(N, st, 4, 2, N->p2, N->a2, N->gB[2], N->gA[2]); // dP2 (32 ch) overwrites
  float *dS1 = N->gA[1] + 64 * V1;
  note_launch();
  k_pool_back_add<<<line_blocks(32, d[1].Z, d[1].Y), 128, 0, st>>>(d[1], d[2], 32, N->gA[2], dS1);
  conv_back(N, st, 3, 1, N->a1, N->c1 + 64 * V1, dS1, N->gB[1]);
  conv_back(N, st, 2, 1, N->p1, N->a1, N->gB[1], N->gA[1]);
  float *dS0 = N->gA[0] + 32 * V0;
  note_launch();
  k_pool_back_add<<<line_blocks(16, d[0].Z, d[0].Y), 128, 0, st>>>(d[0], d[1], 16, N->gA[1], dS0);
  conv_back(N, st, 1, 0, N->a0, N->c0 + 32 * V0, dS0, N->gB[0]);
  conv_back(N, st, 0, 0, N->in, N->a0, N->gB[0], nullptr);
}

// input scale: the L2 norm over the free DOFs (a point load becomes a unit spike)
double host_norm_free(const icarat_ctx *c, const double *f)
{
  double s = 0.0;
  for(int i = 0; i < c->numeq; i++)
    s += f[i] * f[i];
  s = std::sqrt(s);
  return s > 0.0 ? s : 1.0;
}

} // namespace

namespace icarat_b200
{
// z = s * net(r / s) on ctx's grid and design (r: full node vector of T).
template <typename T>
void net_apply(icarat_net *N, icarat_ctx *c, const T *r, double s, T *z)
{
  ensure_grid(N, c);
  refresh_weights(N, c->stream);
  const GridDev g{c->nx, c->ny, c->nz, c->NX, c->NY, c->NZ, c->numnp, c->nelx};
  note_launch();
  k_net_input<T><<<nb(N->d[0].V), 256, 0, c->stream>>>(N->d[0], g, r, c->d_fix, c->d_rho,
                                                       (float)(1.0 / s), N->in);
  forward(N, c->stream);
  note_launch();
  k_net_output<T><<<nb(c->numnp), 256, 0, c->stream>>>(N->d[0], g, N->out, c->d_fix, s, z);
  ICK(cudaGetLastError());
}
void net_check(icarat_net *N, cudaStream_t st) { check_tc_conv(N, st); }

template void net_apply<float>(icarat_net *, icarat_ctx *, const float *, double, float *);
template void net_apply<double>(icarat_net *, icarat_ctx *, const double *, double, double *);
} // namespace icarat_b200

extern "C" {

int icarat_net_create(int device, unsigned long long seed, icarat_net **out)
{
  ICARAT_API_BEGIN
  IREQUIRE(out, ICARAT_ERR_ARG, "null argument");
  *out = nullptr;
  ICK(cudaSetDevice(device));
  icarat_net *N = new icarat_net;
  N->device = device;
  long o = 0;
  for(int l = 0; l < 15; l++)
  {
    NetLayer &Ly = N->L[l];
    Ly.cin = kLayers[l][0];
    Ly.cout = kLayers[l][1];
    Ly.k = kLayers[l][2];
    Ly.woff = o;
    o += (long)Ly.cout * Ly.cin * Ly.k * Ly.k * Ly.k;
    Ly.boff = o;
    o += Ly.cout;
    N->lt.cin[l] = Ly.cin;
    N->lt.cout[l] = Ly.cout;
    N->lt.k[l] = Ly.k;
    N->lt.woff[l] = Ly.woff;
    N->lt.boff[l] = Ly.boff;
  }
  N->np = o;
  try
  {
    // He-normal weights (the head scaled by 0.1), zero biases
    std::vector<float> w(o, 0.0f);
    std::mt19937_64 gen(seed);
    std::normal_distribution<double> nd(0.0, 1.0);
    for(int l = 0; l < 15; l++)
    {
      const NetLayer &Ly = N->L[l];
      const long nw = (long)Ly.cout * Ly.cin * Ly.k * Ly.k * Ly.k;
      const double sd = std::sqrt(2.0 / (Ly.cin * Ly.k * Ly.k * Ly.k)) * (l == 14 ? 0.1 : 1.0);
      for(long i = 0; i < nw; i++)
        w[Ly.woff + i] = (float)(sd * nd(gen));
    }
    N->w = alloc_n<float>(o);
    N->m = alloc_n<float>(o);
    N->v = alloc_n<float>(o);
    N->g = alloc_n<float>(o);
    N->wb = alloc_n<bf16>(o);
    N->wt = alloc_n<bf16>(o);
    long po = 0;
    for(int l = 0; l < 15; l++)
      if(N->L[l].k == 3)
      {
        N->wpk_off[l] = po;
        po += conv3_tc_packed_size(N->L[l].cin, N->L[l].cout);
      }
    N->wpk = alloc_n<bf16>(po);
    N->tc_err = alloc_n<int>(1);
    ICK(cudaMemset(N->tc_err, 0, sizeof(int)));
    ICK(cudaMemcpy(N->w, w.data(), sizeof(float) * o, cudaMemcpyHostToDevice));
    ICK(cudaMemset(N->m, 0, sizeof(float) * o));
    ICK(cudaMemset(N->v, 0, sizeof(float) * o));
    ICK(cudaMemset(N->g, 0, sizeof(float) * o));
    ICK(cudaMallocHost(&N->h_lpart, sizeof(double) * 3 * 4096));
  }
  catch(...)
  {
    icarat_net_destroy(N);
    throw;
  }
  *out = N;
  return ICARAT_OK;
  ICARAT_API_END
}

int icarat_net_destroy(icarat_net *N)
{
  if(!N)
    return ICARAT_OK;
  cudaSetDevice(N->device);
  cudaDeviceSynchronize();
  free_acts(N);
  for(void *p : {(void *)N->w, (void *)N->m, (void *)N->v, (void *)N->g, (void *)N->wb,
                 (void *)N->wt, (void *)N->wpk, (void *)N->tc_err})
    if(p)
      cudaFree(p);
  if(N->h_lpart)
    cudaFreeHost(N->h_lpart);
  delete N;
  return ICARAT_OK;
}

int icarat_net_num_params(icarat_net *N, long long *n)
{
  ICARAT_API_BEGIN
  IREQUIRE(N && n, ICARAT_ERR_ARG, "null argument");
  *n = N->np;
  return ICARAT_OK;
  ICARAT_API_END
}

int icarat_net_get_params(icarat_net *N, float *w)
{
  ICARAT_API_BEGIN
  IREQUIRE(N && w, ICARAT_ERR_ARG, "null argument");
  ICK(cudaDeviceSynchronize());
  ICK(cudaMemcpy(w, N->w, sizeof(float) * N->np, cudaMemcpyDeviceToHost));
  return ICARAT_OK;
  ICARAT_API_END
}

int icarat_net_set_params(icarat_net *N, const float *w)
{
  ICARAT_API_BEGIN
  IREQUIRE(N && w, ICARAT_ERR_ARG, "null argument");
  ICK(cudaDeviceSynchronize());
  ICK(cudaMemcpy(N->w, w, sizeof(float) * N->np, cudaMemcpyHostToDevice));
  ICK(cudaMemset(N->m, 0, sizeof(float) * N->np));
  ICK(cudaMemset(N->v, 0, sizeof(float) * N->np));
  N->step = 0;
  N->wdirty = true;
  return ICARAT_OK;
  ICARAT_API_END
}

int icarat_net_get_grads(icarat_net *N, float *g)
{
  ICARAT_API_BEGIN
  IREQUIRE(N && g, ICARAT_ERR_ARG, "null argument");
  ICK(cudaDeviceSynchronize());
  ICK(cudaMemcpy(g, N->g, sizeof(float) * N->np, cudaMemcpyDeviceToHost));
  return ICARAT_OK;
  ICARAT_API_END
}

int icarat_net_train_step(icarat_net *N, icarat_ctx *c, const double *rho, const double *f,
                          const double *u, double lr, double *loss)
{
  ICARAT_API_BEGIN
  IREQUIRE(c == nullptr || !c->sel, ICARAT_ERR_UNSUPPORTED,
           "the learned preconditioner is not available on a selected (sub-)mesh");
  IREQUIRE(N && c && rho && f && u, ICARAT_ERR_ARG, "null argument");
  IREQUIRE(lr >= 0.0, ICARAT_ERR_ARG, "learning rate must be >= 0");
  ICK(cudaSetDevice(c->device));
  ensure_grid(N, c);
  refresh_weights(N, c->stream);
  cudaStream_t st = c->stream;
  const GridDev g{c->nx, c->ny, c->nz, c->NX, c->NY, c->NZ, c->numnp, c->nelx};
  const double s = host_norm_free(c, f);
  // sample on the device: rho -> d_e1, f -> d_Ap, u -> d_z (full vectors)
  ICK(cudaMemcpyAsync(c->d_e1, rho, sizeof(double) * c->nelx, cudaMemcpyHostToDevice, st));
  to_full(c, f, c->d_Ap, true);
  to_full(c, u, c->d_z, true);
  const Dims &d0 = N->d[0];
  note_launch(2);
  k_net_input<double><<<nb(d0.V), 256, 0, st>>>(d0, g, c->d_Ap, c->d_fix, c->d_e1,
                                               (float)(1.0 / s), N->in);
  k_net_target<<<nb(d0.V), 256, 0, st>>>(d0, g, c->d_z, c->d_fix, 1.0 / s, N->tgt, N->mask);
  forward(N, st);
  const long n3 = 3 * d0.V;
  const int lb = std::min(nb(n3), 4096);
  note_launch();
  k_net_loss<<<lb, 256, 0, st>>>(n3, N->out, N->tgt, N->mask, N->lpart);
  ICK(cudaMemcpyAsync(N->h_lpart, N->lpart, sizeof(double) * 3 * lb, cudaMemcpyDeviceToHost, st));
  ICK(cudaStreamSynchronize(st));
  double A = 0.0, Y = 0.0, T = 0.0;
  for(int b = 0; b < lb; b++)
  {
    A += N->h_lpart[3 * b];
    Y += N->h_lpart[3 * b + 1];
    T += N->h_lpart[3 * b + 2];
  }
  IREQUIRE(T > 0.0, ICARAT_ERR_ARG, "training target is zero");
  IREQUIRE(A == A && Y == Y, ICARAT_ERR_NAN, "non-finite network output");
  Y += 1e-30;
  // 1 - cos^2 plus kNetNormPenalty (|y|^2 - 1)^2, which keeps the otherwise
  // free output scale near 1
  if(loss)
    *loss = 1.0 - A * A / (Y * T) + kNetNormPenalty * (Y - 1.0) * (Y - 1.0);
  note_launch();
  k_net_dout<<<nb(n3), 256, 0, st>>>(
      n3, N->out, N->tgt, N->mask, (float)(-2.0 * A / (Y * T)),
      (float)(2.0 * A * A / (Y * Y * T) + 4.0 * kNetNormPenalty * (Y - 1.0)), N->dout);
  backward(N, st);
  if(lr > 0.0)
  {
    N->step++;
    const double b1 = 0.9, b2 = 0.999;
    const double c1 = 1.0 - std::pow(b1, (double)N->step), c2 = 1.0 - std::pow(b2, (double)N->step);
    note_launch();
    k_adam<<<nb(N->np), 256, 0, st>>>(N->np, N->w, N->m, N->v, N->g, (float)lr, (float)b1,
                                      (float)b2, (float)c1, (float)c2, 1e-8f);
    N->wdirty = true;
  }
  check_tc_conv(N, st);
  return ICARAT_OK;
  ICARAT_API_END
}

int icarat_net_infer(icarat_net *N, icarat_ctx *c, const double *f, double *u)
{
  ICARAT_API_BEGIN
  IREQUIRE(N && c && f && u, ICARAT_ERR_ARG, "null argument");
  IREQUIRE(c->design_set, ICARAT_ERR_STATE, "set the design first");
  ICK(cudaSetDevice(c->device));
  const double s = host_norm_free(c, f);
  to_full(c, f, c->d_Ap, true);
  net_apply<double>(N, c, c->d_Ap, s, c->d_z);
  check_tc_conv(N, c->stream);
  from_full(c, c->d_z, u, true);
  return ICARAT_OK;
  ICARAT_API_END
}

int icarat_net_infer_dev(icarat_net *N, icarat_ctx *c, const double *f, double *u)
{
  ICARAT_API_BEGIN
  IREQUIRE(N && c && f && u, ICARAT_ERR_ARG, "null argument");
  IREQUIRE(c->design_set, ICARAT_ERR_STATE, "set the design first");
  ICK(cudaSetDevice(c->device));
  to_full(c, f, c->d_Ap, false);
  const double bb = device_dot(c, c->d_Ap, c->d_Ap, c->neq);
  net_apply<double>(N, c, c->d_Ap, bb > 0.0 ? std::sqrt(bb) : 1.0, c->d_z);
  check_tc_conv(N, c->stream);
  from_full(c, c->d_z, u, false);
  return ICARAT_OK;
  ICARAT_API_END
}

int icarat_ctx_set_net(icarat_ctx *c, icarat_net *N)
{
  ICARAT_API_BEGIN
  IREQUIRE(c == nullptr || !c->sel, ICARAT_ERR_UNSUPPORTED,
           "the learned preconditioner is not available on a selected (sub-)mesh");
  IREQUIRE(c, ICARAT_ERR_ARG, "null context");
  c->net = N;
  return ICARAT_OK;
  ICARAT_API_END
}

} // extern "C"
