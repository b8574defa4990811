// Dense FP64 linear algebra for the coarsest multigrid level, on the FP64
// tensor cores (mma.sync m8n8k4 f64, the DMMA path of sm_100a).
//
// The coarsest operator A (n x n SPD, n = free DOFs of the coarsest grid)
// changes with every design, so each design computes W = L^-1 of its
// Cholesky factor A = L L^T, and every V-cycle solves A x = b as
// x = W^T (W b) with two triangular matrix-vector products.
//   1. right-looking blocked Cholesky, block 64: per block k the diagonal
//      block is factored and inverted in registers (k_potrf64, which also
//      stores W_kk = L_kk^-1), the panel becomes L_ik = A_ik W_kk^T and the
//      trailing matrix takes A -= L_ik L_jk^T (lower tiles), both as GEMMs
//      limited to the matrix's band (the caller orders the unknowns so that
//      the band is narrow);
//   2. W by triangular inversion in doubling steps: with L = [L11 0; L21 L22],
//      W21 = -W22 (L21 W11), two batched GEMMs per block size over the band
//      of L21.
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
  // batch (grid z): product z uses A + z za, B + z zb, C + z zc; with
  // rows0 > 0 it has at most rows0 - z rows_step rows (and, with k_clip, at
  // most that many terms)
  long za, zb, zc;
  int rows0, rows_step, k_clip;
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
  chain_wait();
  const int tm = blockIdx.y, tn = blockIdx.x;
  if(g.lower && tn > tm)
    return;
  if(blockIdx.z > 0)
  {
    g.A += blockIdx.z * g.za;
    g.B += blockIdx.z * g.zb;
    g.C += blockIdx.z * g.zc;
  }
  if(g.rows0 > 0)
  {
    const int rows = g.rows0 - (int)blockIdx.z * g.rows_step;
    g.M = min(g.M, rows);
    if(g.k_clip)
      g.K = min(g.K, rows);
  }
  if(tm * 64 >= g.M)
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
// 4ty..4ty+3 and columns 4tx..4tx+3 of the block (a) and of the inverse being
// built (e).  Elimination is right-looking in the unscaled form: step j
// subtracts m_rj = a_rj / a_jj times row j from every row r > j, both in a
// (a_rc -= m_rj a_cj, lower part) and in e, which starts as the identity
// (e_rc -= m_rj e_jc, c <= j), so that e ends as the inverse of the unit
// lower factor; the square roots of the pivots scale both at the end
// (L_rc = a_rc / sqrt(a_cc), W_rc = e_rc / sqrt(a_rr)).  Column j of a, row
// j of e and 1 / a_jj are final after step j - 1: their owners publish them
// to shared memory at the end of that step (the pivot's owner updates it
// and starts its reciprocal before its other updates), double-buffered, so
// each step needs a single barrier.
constexpr int kPotrfSmem = (4 * 64 + 2 * 64 + 2) * sizeof(double);

// 1 / x and 1 / sqrt(x) for x > 0 by Newton's method from an FP32 seed
// (y <- y (2 - x y), and y <- y (3/2 - x y^2 / 2)): each step doubles the
// correct digits, so two steps take the seed's ~2^-22 past double precision
// (x must lie in the normal FP32 range).  Inline FMAs only: an out-of-line
// divide or square root inside the loops below would save the
// register-resident block to the stack at every call.
__device__ __forceinline__ double recip_newton(double x)
{
  double y = (double)__fdividef(1.0f, (float)x);
#pragma unroll
  for(int it = 0; it < 2; it++)
    y = y * fma(-x, y, 2.0);
  return y;
}

__device__ __forceinline__ double rsqrt_newton(double x)
{
  double y = (double)rsqrtf((float)x);
#pragma unroll
  for(int it = 0; it < 2; it++)
    y = y * fma(-0.5 * x, y * y, 1.5);
  return y;
}

__global__ void __launch_bounds__(256) k_potrf64(double *A, double *W, int n, int k0)
{
  chain_wait();
  extern __shared__ double potrf_smem[];
  double(*colbuf)[64] = reinterpret_cast<double(*)[64]>(potrf_smem); // [2][64] column j of a
  double(*rowbuf)[64] = colbuf + 2;                                  // [2][64] row j of e
  double *isq = potrf_smem + 4 * 64;                                  // 1 / sqrt(pivot)
  double *sq = isq + 64;                                              // sqrt(pivot)
  double *invbuf = sq + 64;                                           // [2] 1 / a_jj
  const int t = threadIdx.x, tx = t & 15, ty = t >> 4;
  const int m = min(64, n - k0);
  double a[4][4], e[4][4];
#pragma unroll
  for(int i = 0; i < 4; i++)
#pragma unroll
    for(int q = 0; q < 4; q++)
    {
      const int r = 4 * ty + i, c = 4 * tx + q;
      a[i][q] = (r < m && c < m) ? A[(long)(k0 + r) * n + k0 + c] : (r == c ? 1.0 : 0.0);
      e[i][q] = (r == c) ? 1.0 : 0.0;
    }
  if(tx == 0)
#pragma unroll
    for(int i = 0; i < 4; i++)
      colbuf[0][4 * ty + i] = a[i][0];
  if(ty == 0)
#pragma unroll
    for(int q = 0; q < 4; q++)
      rowbuf[0][4 * tx + q] = e[0][q];
  if(t == 0)
    invbuf[0] = recip_newton(a[0][0]);
  __syncthreads();
  auto step = [&](auto qc, int j)
  {
    constexpr int Q = decltype(qc)::value; // j & 3
    constexpr int Q1 = (Q + 1) & 3;        // (j + 1) & 3
    const double *cj = colbuf[j & 1];
    const double *ej = rowbuf[j & 1];
    const double inv = invbuf[j & 1];
    // multipliers zero outside the rows / columns that step j updates, so
    // that every update below is unconditional: rows r > j of a (columns
    // c > j; the entries above the diagonal follow the symmetric update and
    // are never output) and of e (row j of e is zero past column j)
    double fr[4], fc[4], er[4];
#pragma unroll
    for(int i = 0; i < 4; i++)
    {
      fr[i] = (4 * ty + i > j) ? cj[4 * ty + i] * inv : 0.0; // m_rj
      fc[i] = (4 * tx + i > j) ? cj[4 * tx + i] : 0.0;       // a_cj
      er[i] = ej[4 * tx + i];                                // e_jc
    }
    const int j1 = j + 1;
    // the next pivot's reciprocal, computed by every thread without a branch
    // (only the pivot's owner publishes it) so that its latency hides behind
    // the independent updates below
    const bool pivot_owner = (tx == (j1 >> 2)) && (ty == (j1 >> 2)) && j1 < 64;
    const double inv_next = recip_newton(fma(-fr[Q1], fc[Q1], a[Q1][Q1]));
#pragma unroll
    for(int i = 0; i < 4; i++)
#pragma unroll
      for(int q = 0; q < 4; q++)
      {
        a[i][q] = fma(-fr[i], fc[q], a[i][q]);
        e[i][q] = fma(-fr[i], er[q], e[i][q]);
      }
    if(j1 < 64)
    {
      if(tx == (j1 >> 2))
#pragma unroll
        for(int i = 0; i < 4; i++)
          colbuf[j1 & 1][4 * ty + i] = a[i][Q1];
      if(ty == (j1 >> 2))
#pragma unroll
        for(int q = 0; q < 4; q++)
          rowbuf[j1 & 1][4 * tx + q] = e[Q1][q];
      if(pivot_owner)
        invbuf[j1 & 1] = inv_next;
    }
    __syncthreads();
  };
  for(int j = 0; j < 64; j += 4)
  {
    step(std::integral_constant<int, 0>{}, j);
    step(std::integral_constant<int, 1>{}, j + 1);
    step(std::integral_constant<int, 2>{}, j + 2);
    step(std::integral_constant<int, 3>{}, j + 3);
  }
  // ---- scaling by the square roots of the pivots
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
      if(r < m && c < m)
      {
        A[(long)(k0 + r) * n + k0 + c] = r > c ? a[i][q] * isq[c] : (r == c ? sq[c] : 0.0);
        W[(long)(k0 + r) * n + k0 + c] = (c <= r) ? e[i][q] * isq[r] : 0.0;
      }
    }
}

// The row a warp takes in the triangular products: even warps the short
// rows from the top, odd warps the long ones from the bottom, so every pair
// of neighbouring warps reads n + 1 coefficients and the blocks stay balanced.
__device__ __forceinline__ int trmv_row(int warp, int n)
{
  return (warp & 1) ? n - 1 - (warp >> 1) : (warp >> 1);
}

// sum over q in [q0, q1) of row[q] v[q] by one warp: eight independent
// partial sums per lane (eight coefficient loads in flight), summed in a
// fixed order, then across the warp
__device__ __forceinline__ double warp_row_dot(const double *__restrict__ row,
                                               const double *__restrict__ v, int q0, int q1,
                                               int lane)
{
  double s[8];
#pragma unroll
  for(int u = 0; u < 8; u++)
    s[u] = 0.0;
  int q = q0 + lane;
  for(; q + 224 < q1; q += 256)
#pragma unroll
    for(int u = 0; u < 8; u++)
      s[u] = fma(row[q + 32 * u], v[q + 32 * u], s[u]);
  for(; q < q1; q += 32)
    s[0] = fma(row[q], v[q], s[0]);
  double a = ((s[0] + s[1]) + (s[2] + s[3])) + ((s[4] + s[5]) + (s[6] + s[7]));
  for(int o = 16; o > 0; o >>= 1)
    a += __shfl_down_sync(0xffffffffu, a, o);
  return a;
}

// t = W v (W lower triangular), one warp per row
__global__ void k_trmv_lower(int n, const double *__restrict__ W,
                             const double *__restrict__ v, double *__restrict__ t,
                             const int *__restrict__ halt)
{
  chain_wait();
  if(halted(halt))
    return;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  for(int w = warp; w < n; w += nw)
  {
    const int r = trmv_row(w, n);
    const double s = warp_row_dot(W + (long)r * n, v, 0, r + 1, lane);
    if(lane == 0)
      t[r] = s;
  }
}

// WT = W^T (W lower -> WT upper), 32 x 32 tiles through shared memory
__global__ void k_transpose_lower(int n, const double *__restrict__ W,
                                  double *__restrict__ WT)
{
  chain_wait();
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
                             double *__restrict__ x, const int *__restrict__ halt)
{
  chain_wait();
  if(halted(halt))
    return;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  for(int w = warp; w < n; w += nw)
  {
    const int r = trmv_row(w, n);
    const double s = warp_row_dot(WT + (long)r * n, t, r, n, lane);
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
             B,   ldb, tb, C,    ldc,  lower, a_lower, b_lower, 0, 0, 0, 0, 0, 0};
  dim3 grid((N + 63) / 64, (M + 63) / 64);
  note_launch();
  launch_chained(k_gemm_f64, grid, 128, 0, st, g);
}

// W = L^-1 from the diagonal blocks W_kk by doubling: at block size s every
// pair of neighbouring inverted blocks [o, o + s), [o + s, o + 2s) (o a
// multiple of 2s; the second may be short or absent) becomes one, with
// L = [L11 0; L21 L22], W21 = -W22 L21 W11.  All pairs of one size go in one
// batched launch per product.  L has lower bandwidth bw, so L21 is zero
// outside its top-right min(bw, s2) x min(bw, s) corner:
//   T = L21[0:r, s-k:s] W11[s-k:s, :]   (r x s; the other rows are zero)
//   W21 = -W22[:, 0:r] T                (columns past each row of the lower
//                                        triangular W22 skipped)
// T holds one r x s slab per pair.
static void trinv_banded(cudaStream_t st, const double *L, double *W, double *T, int n,
                         int bw)
{
  for(int s = 64; s < n; s *= 2)
  {
    const int pairs = (n - s + 2 * s - 1) / (2 * s); // pairs whose second block exists
    const int k = std::min(bw, s);
    const int r = std::min(bw, s);
    const long step = 2L * s * n + 2L * s;           // from pair z to pair z + 1
    const long tslab = (long)r * s;
    note_launch(2);
    // T_z = L21 W11 (rows clipped to the short second block of the last pair)
    GemmArgs g1{r, s, k, 1.0, 0.0, L + (long)s * n + s - k, n, 0, W + (long)(s - k) * n, n, 0,
                T, s, 0, 0, 0, step, step, tslab, n - s, 2 * s, 0};
    launch_chained(k_gemm_f64, dim3((s + 63) / 64, (r + 63) / 64, pairs), 128, 0, st, g1);
    // W21_z = -W22 T_z (K clipped like the rows: W22 has s2 columns)
    GemmArgs g2{s, s, r, -1.0, 0.0, W + (long)s * n + s, n, 0, T, s, 0, W + (long)s * n, n,
                0, 1, 0, step, tslab, step, n - s, 2 * s, 1};
    launch_chained(k_gemm_f64, dim3((s + 63) / 64, (s + 63) / 64, pairs), 128, 0, st, g2);
  }
}

// A (lower part, lower bandwidth bw) -> L in place; W <- L^-1 (upper part
// zero); T: n x n scratch, which ends up holding W^T (upper part; rows
// contiguous for the transposed product of every solve).  The Cholesky
// factor keeps the band, so block column k updates only the bw rows below
// its diagonal block; W = L^-1 is dense.
void dense_spd_inverse_factor(cudaStream_t st, double *A, double *W, double *T, int n, int bw)
{
  ICK(cudaFuncSetAttribute(k_potrf64, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           kPotrfSmem));
  ICK(cudaMemsetAsync(W, 0, sizeof(double) * (size_t)n * n, st));
  bw = std::max(1, std::min(bw, n));
  const int nb = (n + 63) / 64;
  for(int k = 0; k < nb; k++)
  {
    const int k0 = k * 64;
    note_launch();
    launch_chained(k_potrf64, 1, 256, kPotrfSmem, st, A, W, n, k0);
    const int rest = std::min(n - k0 - 64, bw);
    if(rest > 0)
    {
      double *panel = A + (long)(k0 + 64) * n + k0;
      // L_ik = A_ik W_kk^T (in place: each CTA reads its own rows first)
      gemm(st, rest, 64, 64, 1.0, panel, n, 0, W + (long)k0 * n + k0, n, 1, 0.0, panel, n,
           0);
      // A22 -= L_i L_j^T on the lower tiles of the band
      gemm(st, rest, rest, 64, -1.0, panel, n, 0, panel, n, 1, 1.0,
           A + (long)(k0 + 64) * n + k0 + 64, n, 1);
    }
  }
  trinv_banded(st, A, W, T, n, bw);
  note_launch();
  launch_chained(k_transpose_lower, dim3((n + 31) / 32, (n + 31) / 32), dim3(32, 8), 0, st, n,
                 (const double *)W, T);
  ICK(cudaGetLastError());
}

// x[rowmap] = W^T W b[rowmap]  (WT = W^T from dense_spd_inverse_factor); both
// products return at entry while *halt != 0 (halt null: never)
void dense_spd_solve(cudaStream_t st, const double *W, const double *WT, int n,
                     const double *v, double *t, const int *rowmap, double *x,
                     const int *halt)
{
  note_launch(2);
  const int blocks = (n * 32 + 255) / 256;
  launch_chained(k_trmv_lower, blocks, 256, 0, st, n, W, v, t, halt);
  launch_chained(k_trmv_upper, blocks, 256, 0, st, n, WT, t, rowmap, x, halt);
}

} // namespace icarat_b200
