// Dense FP64 linear algebra for the coarsest multigrid level, on the FP64
// tensor cores (mma.sync m8n8k4 f64, the DMMA path of sm_100a).
//
// The coarsest operator A (n x n SPD, n = free DOFs of the coarsest grid)
// changes with every design, so each design computes W = L^-1 of its
// Cholesky factor A = L L^T, and every V-cycle solves A x = b as
// x = W^T (W b) with two triangular matrix-vector products.
//   1. right-looking blocked Cholesky, block 64: per block k the diagonal
//      block is factored and inverted in shared memory (k_potrf64, which also
//      stores W_kk = L_kk^-1), the panel becomes L_ik = A_ik W_kk^T and the
//      trailing matrix takes A -= L_ik L_jk^T (lower tiles), both as GEMMs;
//   2. W by recursive triangular inversion: with L = [L11 0; L21 L22],
//      W21 = -W22 (L21 W11), two GEMMs per split.
// Matrices are row-major with leading dimension n.
#include <type_traits>

#include "internal.cuh"

namespace icarat_b200
{

__device__ __forceinline__ void dmma884(double (&d)[2], double a, double b)
{
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, "
               "{%0,%1};\n"
               : "+d"(d[0]), "+d"(d[1])
               : "d"(a), "d"(b));
}

// C(i,j) = alpha sum_k op(A)(i,k) op(B)(k,j) + beta C(i,j) for i < M, j < N.
// op(A)(i,k) = ta ? A[k lda + i] : A[i lda + k]; op(B)(k,j) = tb ? B[j ldb + k]
// : B[k ldb + j].  lower != 0: only tiles / elements with j <= i.
struct GemmArgs
{
  int M, N, K;
  double alpha, beta;
  const double *A;
  long lda;
  int ta;
  const double *B;
  long ldb;
  int tb;
  double *C;
  long ldc;
  int lower;
  int a_lower; // op(A)(i,k) = 0 for k > i: K ends at the tile's last row
  int b_lower; // op(B)(k,j) = 0 for k < j: K starts at the tile's first column
};

// Element t of a 64 x 16 A chunk / 16 x 64 B chunk, ordered so that the
// stored (contiguous) axis runs across consecutive threads.
__device__ __forceinline__ void gemm_a_idx(int ta, int t, int &r, int &c)
{
  if(ta)
  {
    c = t >> 6;
    r = t & 63;
  }
  else
  {
    r = t >> 4;
    c = t & 15;
  }
}
__device__ __forceinline__ void gemm_b_idx(int tb, int t, int &kr, int &jc)
{
  if(tb)
  {
    jc = t >> 4;
    kr = t & 15;
  }
  else
  {
    kr = t >> 6;
    jc = t & 63;
  }
}

// 64 x 64 tile per CTA, 4 warps of 32 x 32, K staged by 16 in shared memory;
// the next chunk is fetched into registers while the current one is used.
__global__ void __launch_bounds__(128) k_gemm_f64(GemmArgs g)
{
  const int tm = blockIdx.y, tn = blockIdx.x;
  if(g.lower && tn > tm)
    return;
  __shared__ double As[64][16 + 2];
  __shared__ double Bs[16][64 + 2];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wm = warp >> 1, wn = warp & 1;
  double acc[4][4][2];
#pragma unroll
  for(int a = 0; a < 4; a++)
#pragma unroll
    for(int b = 0; b < 4; b++)
      acc[a][b][0] = acc[a][b][1] = 0.0;
  const int i0 = tm * 64, j0 = tn * 64;
  const int kb = g.b_lower ? (j0 & ~15) : 0;
  const int ke = g.a_lower ? min(g.K, i0 + 64) : g.K;
  double ra[8], rb[8];
  auto fetch = [&](int k0)
  {
#pragma unroll
    for(int u = 0; u < 8; u++)
    {
      const int t = threadIdx.x + 128 * u;
      int r, c, kr, jc;
      gemm_a_idx(g.ta, t, r, c);
      gemm_b_idx(g.tb, t, kr, jc);
      const int gi = i0 + r, gk = k0 + c;
      ra[u] = (gi < g.M && gk < g.K)
                  ? (g.ta ? g.A[(long)gk * g.lda + gi] : g.A[(long)gi * g.lda + gk])
                  : 0.0;
      const int bk = k0 + kr, bj = j0 + jc;
      rb[u] = (bk < g.K && bj < g.N)
                  ? (g.tb ? g.B[(long)bj * g.ldb + bk] : g.B[(long)bk * g.ldb + bj])
                  : 0.0;
    }
  };
  if(kb < ke)
    fetch(kb);
  for(int k0 = kb; k0 < ke; k0 += 16)
  {
#pragma unroll
    for(int u = 0; u < 8; u++)
    {
      const int t = threadIdx.x + 128 * u;
      int r, c, kr, jc;
      gemm_a_idx(g.ta, t, r, c);
      gemm_b_idx(g.tb, t, kr, jc);
      As[r][c] = ra[u];
      Bs[kr][jc] = rb[u];
    }
    __syncthreads();
    if(k0 + 16 < ke)
      fetch(k0 + 16);
#pragma unroll
    for(int kk = 0; kk < 16; kk += 4)
    {
      double a[4], b[4];
#pragma unroll
      for(int mt = 0; mt < 4; mt++)
        a[mt] = As[wm * 32 + mt * 8 + (lane >> 2)][kk + (lane & 3)];
#pragma unroll
      for(int nt = 0; nt < 4; nt++)
        b[nt] = Bs[kk + (lane & 3)][wn * 32 + nt * 8 + (lane >> 2)];
#pragma unroll
      for(int mt = 0; mt < 4; mt++)
#pragma unroll
        for(int nt = 0; nt < 4; nt++)
          dmma884(acc[mt][nt], a[mt], b[nt]);
    }
    __syncthreads();
  }
#pragma unroll
  for(int mt = 0; mt < 4; mt++)
#pragma unroll
    for(int nt = 0; nt < 4; nt++)
#pragma unroll
      for(int q = 0; q < 2; q++)
      {
        const int i = i0 + wm * 32 + mt * 8 + (lane >> 2);
        const int j = j0 + wn * 32 + nt * 8 + 2 * (lane & 3) + q;
        if(i < g.M && j < g.N && (!g.lower || j <= i))
        {
          double *c = g.C + (long)i * g.ldc + j;
          const double v = g.alpha * acc[mt][nt][q];
          *c = (g.beta != 0.0) ? v + g.beta * *c : v;
        }
      }
}

// Factor the 64 x 64 diagonal block at k0, write L_kk into A (zeros above the
// diagonal) and W_kk = L_kk^-1 into W.  Rows / columns past n are padded with
// the identity.
//
// The block lives in registers: thread (ty, tx) of a 16 x 16 grid holds rows
// 4ty..4ty+3 and columns 4tx..4tx+3.  Elimination is right-looking in the
// unscaled form a_rc -= a_rj a_cj / a_jj (the square roots and the column
// scaling come after the loop): per column j the owners publish column j to
// shared memory and one barrier later every thread updates its 16 entries.
// The inverse is a forward substitution by rows in the same tiles (row k of
// L^-1 and column k of L published per step).  The published vectors are
// double-buffered, so each step needs a single barrier.
constexpr int kPotrfSmem = (4 * 64 + 2 * 64) * sizeof(double);

// 1 / x and 1 / sqrt(x) for x > 0 by Newton's method from an FP32 seed
// (y <- y (2 - x y), and y <- y (3/2 - x y^2 / 2)): each step doubles the
// correct digits, three steps reach double precision from the seed's ~2^-22.
// Inline FMAs only: an out-of-line divide or square root inside the loops
// below would save the register-resident block to the stack at every call.
__device__ __forceinline__ double recip_newton(double x)
{
  double y = (double)__fdividef(1.0f, (float)x);
#pragma unroll
  for(int it = 0; it < 3; it++)
    y = y * fma(-x, y, 2.0);
  return y;
}

__device__ __forceinline__ double rsqrt_newton(double x)
{
  double y = (double)rsqrtf((float)x);
#pragma unroll
  for(int it = 0; it < 3; it++)
    y = y * fma(-0.5 * x, y * y, 1.5);
  return y;
}

__global__ void __launch_bounds__(256) k_potrf64(double *A, double *W, int n, int k0)
{
  extern __shared__ double potrf_smem[];
  double(*vec)[64] = reinterpret_cast<double(*)[64]>(potrf_smem); // [4][64]
  double *isq = potrf_smem + 4 * 64; // 1 / sqrt(pivot)
  double *sq = isq + 64;              // sqrt(pivot)
  const int t = threadIdx.x, tx = t & 15, ty = t >> 4;
  const int m = min(64, n - k0);
  double a[4][4];
#pragma unroll
  for(int i = 0; i < 4; i++)
#pragma unroll
    for(int q = 0; q < 4; q++)
    {
      const int r = 4 * ty + i, c = 4 * tx + q;
      a[i][q] = (r < m && c < m) ? A[(long)(k0 + r) * n + k0 + c] : (r == c ? 1.0 : 0.0);
    }
  // ---- elimination (by 4 columns, so that the published register column is
  // a compile-time index)
  auto elim = [&](auto qc, int j)
  {
    constexpr int Q = decltype(qc)::value;
    double *col = vec[j & 1];
    if(tx == (j >> 2))
#pragma unroll
      for(int i = 0; i < 4; i++)
        col[4 * ty + i] = a[i][Q];
    __syncthreads();
    const double inv = recip_newton(col[j]);
    double fr[4], fc[4];
#pragma unroll
    for(int i = 0; i < 4; i++)
    {
      fr[i] = col[4 * ty + i];
      fc[i] = col[4 * tx + i] * inv;
    }
#pragma unroll
    for(int i = 0; i < 4; i++)
#pragma unroll
      for(int q = 0; q < 4; q++)
      {
        const int r = 4 * ty + i, c = 4 * tx + q;
        if(c > j && r >= c)
          a[i][q] = fma(-fr[i], fc[q], a[i][q]);
      }
  };
  for(int j = 0; j < 64; j += 4)
  {
    elim(std::integral_constant<int, 0>{}, j);
    elim(std::integral_constant<int, 1>{}, j + 1);
    elim(std::integral_constant<int, 2>{}, j + 2);
    if(j + 3 < 63)
      elim(std::integral_constant<int, 3>{}, j + 3);
  }
  // ---- scaling: L_rc = a_rc / sqrt(a_cc), L_cc = sqrt(a_cc)
  if(tx == ty)
#pragma unroll
    for(int i = 0; i < 4; i++)
    {
      const double y = rsqrt_newton(a[i][i]);
      isq[4 * ty + i] = y;
      sq[4 * ty + i] = a[i][i] * y;
    }
  __syncthreads();
#pragma unroll
  for(int i = 0; i < 4; i++)
#pragma unroll
    for(int q = 0; q < 4; q++)
    {
      const int r = 4 * ty + i, c = 4 * tx + q;
      a[i][q] = r > c ? a[i][q] * isq[c] : (r == c ? sq[c] : 0.0);
    }
  // ---- inverse: w = I, then per row k: w_k /= L_kk (final), w_r -= L_rk w_k (r > k)
  double w[4][4];
#pragma unroll
  for(int i = 0; i < 4; i++)
#pragma unroll
    for(int q = 0; q < 4; q++)
      w[i][q] = (4 * ty + i == 4 * tx + q) ? 1.0 : 0.0;
  auto inv_step = [&](auto qc, int k)
  {
    constexpr int Q = decltype(qc)::value;
    double *row = vec[2 + (k & 1)];
    double *colL = vec[k & 1];
    const double ilkk = isq[k]; // 1 / L_kk
    if(ty == (k >> 2))
#pragma unroll
      for(int q = 0; q < 4; q++)
      {
        w[Q][q] *= ilkk;
        row[4 * tx + q] = w[Q][q];
      }
    if(tx == (k >> 2))
#pragma unroll
      for(int i = 0; i < 4; i++)
        colL[4 * ty + i] = a[i][Q];
    __syncthreads();
#pragma unroll
    for(int i = 0; i < 4; i++)
    {
      const int r = 4 * ty + i;
      if(r > k)
      {
        const double l = colL[r];
#pragma unroll
        for(int q = 0; q < 4; q++)
          w[i][q] = fma(-l, row[4 * tx + q], w[i][q]);
      }
    }
  };
  for(int k = 0; k < 64; k += 4)
  {
    inv_step(std::integral_constant<int, 0>{}, k);
    inv_step(std::integral_constant<int, 1>{}, k + 1);
    inv_step(std::integral_constant<int, 2>{}, k + 2);
    inv_step(std::integral_constant<int, 3>{}, k + 3);
  }
#pragma unroll
  for(int i = 0; i < 4; i++)
#pragma unroll
    for(int q = 0; q < 4; q++)
    {
      const int r = 4 * ty + i, c = 4 * tx + q;
      if(r < m && c < m)
      {
        A[(long)(k0 + r) * n + k0 + c] = a[i][q];
        W[(long)(k0 + r) * n + k0 + c] = (c <= r) ? w[i][q] : 0.0;
      }
    }
}

// t = W v (W lower triangular), one warp per row
__global__ void k_trmv_lower(int n, const double *__restrict__ W,
                             const double *__restrict__ v, double *__restrict__ t)
{
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  for(int r = warp; r < n; r += nw)
  {
    const double *row = W + (long)r * n;
    double s = 0.0;
    for(int q = lane; q <= r; q += 32)
      s = fma(row[q], v[q], s);
    for(int o = 16; o > 0; o >>= 1)
      s += __shfl_down_sync(0xffffffffu, s, o);
    if(lane == 0)
      t[r] = s;
  }
}

// WT = W^T (W lower -> WT upper), 32 x 32 tiles through shared memory
__global__ void k_transpose_lower(int n, const double *__restrict__ W,
                                  double *__restrict__ WT)
{
  __shared__ double tile[32][33];
  const int bi = blockIdx.y * 32, bj = blockIdx.x * 32; // source tile rows / cols
  if(bj > bi + 31)
    return; // entirely above the diagonal: zero in W and in WT below
  for(int r = threadIdx.y; r < 32; r += blockDim.y)
  {
    const int i = bi + r, j = bj + threadIdx.x;
    tile[r][threadIdx.x] = (i < n && j < n && j <= i) ? W[(long)i * n + j] : 0.0;
  }
  __syncthreads();
  for(int r = threadIdx.y; r < 32; r += blockDim.y)
  {
    const int i = bj + r, j = bi + threadIdx.x; // WT[i][j] = W[j][i]
    if(i < n && j < n)
      WT[(long)i * n + j] = tile[threadIdx.x][r];
  }
}

// x[rowmap] = WT t (WT upper), one warp per row; rows are contiguous
__global__ void k_trmv_upper(int n, const double *__restrict__ WT,
                             const double *__restrict__ t, const int *__restrict__ rowmap,
                             double *__restrict__ x)
{
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  for(int r = warp; r < n; r += nw)
  {
    const double *row = WT + (long)r * n;
    double s = 0.0;
    for(int q = r + lane; q < n; q += 32)
      s = fma(row[q], t[q], s);
    for(int o = 16; o > 0; o >>= 1)
      s += __shfl_down_sync(0xffffffffu, s, o);
    if(lane == 0)
      x[rowmap[r]] = s;
  }
}


static void gemm(cudaStream_t st, int M, int N, int K, double alpha, const double *A,
                 long lda, int ta, const double *B, long ldb, int tb, double beta,
                 double *C, long ldc, int lower, int a_lower = 0, int b_lower = 0)
{
  if(M <= 0 || N <= 0 || K <= 0)
    return;
  GemmArgs g{M,   N,  K,  alpha, beta, A,     lda,    ta,
             B,   ldb, tb, C,    ldc,  lower, a_lower, b_lower};
  dim3 grid((N + 63) / 64, (M + 63) / 64);
  note_launch();
  k_gemm_f64<<<grid, 128, 0, st>>>(g);
}

// W rows/cols [off, off + nbk * 64) of L^-1, given the diagonal blocks W_kk.
static void trinv_rec(cudaStream_t st, const double *L, double *W, double *T, int n,
                      int off, int nbk)
{
  if(nbk <= 1)
    return;
  const int b1 = nbk / 2, b2 = nbk - b1;
  const int s1 = b1 * 64;
  const int s2 = std::min(b2 * 64, n - off - s1);
  trinv_rec(st, L, W, T, n, off, b1);
  trinv_rec(st, L, W, T, n, off + s1, b2);
  // T = L21 W11  (s2 x s1), then W21 = -W22 T  (s2 x s1)
  // (W11 and W22 are lower triangular: half of each product is skipped)
  gemm(st, s2, s1, s1, 1.0, L + (long)(off + s1) * n + off, n, 0,
       W + (long)off * n + off, n, 0, 0.0, T, s1, 0, 0, 1);
  gemm(st, s2, s1, s2, -1.0, W + (long)(off + s1) * n + off + s1, n, 0, T, s1, 0, 0.0,
       W + (long)(off + s1) * n + off, n, 0, 1, 0);
}

// A (lower part) -> L in place; W <- L^-1 (upper part zero); T: n x n
// scratch, which ends up holding W^T (upper part; rows contiguous for the
// transposed product of every solve).
void dense_spd_inverse_factor(cudaStream_t st, double *A, double *W, double *T, int n)
{
  ICK(cudaFuncSetAttribute(k_potrf64, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           kPotrfSmem));
  ICK(cudaMemsetAsync(W, 0, sizeof(double) * (size_t)n * n, st));
  const int nb = (n + 63) / 64;
  for(int k = 0; k < nb; k++)
  {
    const int k0 = k * 64;
    note_launch();
    k_potrf64<<<1, 256, kPotrfSmem, st>>>(A, W, n, k0);
    const int rest = n - k0 - 64;
    if(rest > 0)
    {
      double *panel = A + (long)(k0 + 64) * n + k0;
      // L_ik = A_ik W_kk^T (in place: each CTA reads its own rows first)
      gemm(st, rest, 64, 64, 1.0, panel, n, 0, W + (long)k0 * n + k0, n, 1, 0.0, panel, n,
           0);
      // A22 -= L_i L_j^T on the lower tiles
      gemm(st, rest, rest, 64, -1.0, panel, n, 0, panel, n, 1, 1.0,
           A + (long)(k0 + 64) * n + k0 + 64, n, 1);
    }
  }
  trinv_rec(st, A, W, T, n, 0, nb);
  note_launch();
  k_transpose_lower<<<dim3((n + 31) / 32, (n + 31) / 32), dim3(32, 8), 0, st>>>(n, W, T);
  ICK(cudaGetLastError());
}

// x[rowmap] = W^T W b[rowmap]  (WT = W^T from dense_spd_inverse_factor)
void dense_spd_solve(cudaStream_t st, const double *W, const double *WT, int n,
                     const double *v, double *t, const int *rowmap, double *x)
{
  note_launch(2);
  k_trmv_lower<<<(n * 32 + 255) / 256, 256, 0, st>>>(n, W, v, t);
  k_trmv_upper<<<(n * 32 + 255) / 256, 256, 0, st>>>(n, WT, t, rowmap, x);
}

} // namespace icarat_b200
