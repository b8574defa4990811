// Element-by-element K u on the 5th-generation tensor cores (tcgen05) in
// BF16 with FP32 accumulation (no reference counterpart; the reference
// assembles K in FP64).
//
// Every element of the uniform voxel mesh shares Ke0, so for 128 elements the
// element products form one GEMM
//     D (128 x 32) = U (128 x 32) Ke0^T (32 x 32),
// U row e = the 24 nodal displacements of element e (DOF 3 a + c, local node
// a, component c), padded to 32 columns; Ke0 padded to 32 x 32.  FP32
// operands are split into BF16 pairs x = hi + lo, and with TERMS = 3 the
// product is U_hi K_hi + U_hi K_lo + U_lo K_hi (about 16 significant bits);
// TERMS = 1 keeps U_hi K_hi only (8 bits).  The moduli E_e scale the rows of
// D in FP32 afterwards.
//
// Tile and sweep.  A CTA of 8 warps owns a column of 31 x 7 nodes (x, y) over
// a range of node layers (z).  Per element layer it multiplies the 32 x 8
// elements around its nodes (one element per thread: x = lane, y = warp; two
// M = 128 MMAs), so every owned node has all 4 elements of the layer inside
// the tile; the one-element halo is recomputed by the neighbouring CTA.  Node
// sums need no atomics: the x pairs are summed by a warp shuffle, the y pairs
// through shared memory and the z pairs in registers carried to the next
// layer.
//
// Pipeline per element layer: the threads gather the next layer's U into the
// other shared-memory stage (BF16 hi/lo in the UMMA K-major core-matrix
// layout, no swizzle) while the tensor core multiplies the current one into
// TMEM; one elected thread issues the MMAs and commits them to an mbarrier;
// the epilogue reads D with tcgen05.ld.  Global loads (displacements one
// layer ahead, moduli and the epilogue's inputs) are issued one iteration
// before their use.  Every wait on an mbarrier is bounded: on expiry the
// kernel records an error and leaves.
#include <cuda_bf16.h>

#include "stencil.cuh"

namespace icarat_b200
{
namespace tc
{

constexpr int kTX = 32, kTY = 8;            // elements per tile row / rows
constexpr int kOX = kTX - 1, kOY = kTY - 1; // owned nodes per layer (x, y)
constexpr int kThreads = kTX * kTY;
constexpr int kMmas = kThreads / 128;       // M = 128 MMAs per layer
constexpr int kK = 32, kN = 32;             // padded element DOFs
constexpr uint32_t kABytes = 128 * kK * 2;  // one M = 128 operand
constexpr uint32_t kBBytes = kN * kK * 2;
constexpr int kTmemCols = 2 * kMmas * 32;   // two stages of 32-column accumulators
constexpr long kWaitLimit = 1L << 24;       // mbarrier polls before giving up

template <int TERMS> struct Smem
{
  alignas(128) uint8_t A[2][kMmas][TERMS == 3 ? 2 : 1][kABytes]; // [stage][mma][hi, lo]
  alignas(128) uint8_t B[2][kBBytes];                            // [hi, lo]
  float xch[2][6][kTY][32];                                      // [stage][dz*3+c][warp][lane]
  double red[32];
  unsigned long long mbar[2];
  uint32_t tmem;
};

// byte offset of the 16-byte row chunk (row r, K chunk kc) in a K-major
// SWIZZLE_NONE operand: core matrices of 8 rows x 16 B, K chunks 128 B apart
// (leading byte offset), 8-row groups 512 B apart (stride byte offset)
__host__ __device__ constexpr uint32_t cm_off(int r, int kc)
{
  return (uint32_t)(((r >> 3) * 4 + kc) * 128 + (r & 7) * 16);
}

__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr)
{
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)(128 >> 4) << 16) |
         ((uint64_t)(512 >> 4) << 32) | (1ull << 46);
}

// kind::f16 instruction descriptor: D F32, A and B BF16, both K-major, N, M
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) |
                            ((uint32_t)(kN >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);

__device__ __forceinline__ uint32_t saddr(const void *p)
{
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void umma(uint32_t d, uint64_t a, uint64_t b, int acc)
{
  asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
               "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d),
               "l"(a), "l"(b), "r"(kIdesc), "r"(acc));
}

__device__ __forceinline__ void umma_commit(uint32_t mbar)
{
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
          mbar)
      : "memory");
}

__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity)
{
  for(long it = 0; it < kWaitLimit; it++)
  {
    uint32_t ok;
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}\n"
                 : "=r"(ok)
                 : "r"(mbar), "r"(parity)
                 : "memory");
    if(ok)
      return true;
  }
  return false;
}

__device__ __forceinline__ void fence_before()
{
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after()
{
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_async_smem()
{
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// the 24 accumulator columns of this thread's TMEM lane
__device__ __forceinline__ void tmem_ld24(uint32_t taddr, float (&v)[24])
{
  uint32_t r[24];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, "
               "%8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
                 "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]),
                 "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
               : "r"(taddr));
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, "
               "[%8];"
               : "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]),
                 "=r"(r[21]), "=r"(r[22]), "=r"(r[23])
               : "r"(taddr + 16u));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for(int q = 0; q < 24; q++)
    v[q] = __uint_as_float(r[q]);
}

__device__ __forceinline__ uint32_t bf2_bits(__nv_bfloat162 h)
{
  return *reinterpret_cast<uint32_t *>(&h);
}

} // namespace tc

template <int OP, int TERMS>
__global__ void __launch_bounds__(tc::kThreads, TERMS == 1 ? 3 : 2) k_ku_tc(TcArgs a)
{
  using namespace tc;
  extern __shared__ __align__(128) uint8_t tc_smem_raw[];
  Smem<TERMS> &sm = *reinterpret_cast<Smem<TERMS> *>(tc_smem_raw);
  chain_wait();
  if(halted(a.halt) || (OP == TC_DOT && a.s->done))
    return;
  const int t = threadIdx.x, w = t >> 5, l = t & 31;
  const GridDev g = a.g;
  const int tile = blockIdx.x;
  const int i0 = (tile % a.tiles_x) * kOX, j0 = (tile / a.tiles_x) * kOY;
  const int kb = blockIdx.y * a.kc;
  const int ke = min(kb + a.kc, g.NZ);
  const int plane = g.NX * g.NY, eplane = g.nx * g.ny, numnp = g.numnp;
  // this thread's element column (x = lane, y = warp) and node column
  const int ei = i0 - 1 + l, ej = j0 - 1 + w;
  const bool e_ok = ei >= 0 && ei < g.nx && ej >= 0 && ej < g.ny;
  const int e_off = ei + ej * g.nx;
  const bool own = l >= 1 && w >= 1 && ei < g.NX && ej < g.NY;
  const int own_off = ei + ej * g.NX;
  bool ld_ok[2], ld1_ok[2];
  int ld_off[2];
#pragma unroll
  for(int dy = 0; dy < 2; dy++)
  {
    const bool yin = ej + dy >= 0 && ej + dy < g.NY;
    ld_ok[dy] = yin && ei >= 0 && ei < g.NX;
    ld1_ok[dy] = yin && l == 31 && ei + 1 < g.NX;
    ld_off[dy] = ei + (ej + dy) * g.NX;
  }
  const int mrow = t & 127, mma = t >> 7; // row of this element in its MMA

  if(t == 0)
  {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(saddr(&sm.mbar[0])), "r"(1));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(saddr(&sm.mbar[1])), "r"(1));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if(w == 0)
  {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     saddr(&sm.tmem)),
                 "r"(kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  // Ke0 hi / lo into the B operand; zero K chunk 3 (columns 24..31) of A
  for(int q = t; q < 2 * kN * 4; q += kThreads)
  {
    const int h = q / (kN * 4), n = (q / 4) % kN, kc = q % 4;
    const uint4 v = *reinterpret_cast<const uint4 *>(a.keb + h * kN * kK + n * kK + kc * 8);
    *reinterpret_cast<uint4 *>(sm.B[h] + cm_off(n, kc)) = v;
  }
#pragma unroll
  for(int s = 0; s < 2; s++)
#pragma unroll
    for(int h = 0; h < (TERMS == 3 ? 2 : 1); h++)
      *reinterpret_cast<uint4 *>(sm.A[s][mma][h] + cm_off(mrow, 3)) = make_uint4(0u, 0u, 0u, 0u);

  // ---- global loads, issued one iteration ahead of their use
  // displacements of node layer k for nodes (ei, ej + dy) (and ei + 1 in
  // lane 31); 32-bit offsets from per-thread bases
  const float *ubase[2][3];
#pragma unroll
  for(int dy = 0; dy < 2; dy++)
#pragma unroll
    for(int c = 0; c < 3; c++)
      ubase[dy][c] = a.u + (c * numnp + ld_off[dy]);
  float pf[2][3], pf1[2][3];
  auto issue_loads = [&](int k)
  {
    const bool kin = k >= 0 && k < g.NZ;
    const int ko = k * plane;
#pragma unroll
    for(int dy = 0; dy < 2; dy++)
    {
      const bool p0 = kin && ld_ok[dy], p1 = kin && ld1_ok[dy];
#pragma unroll
      for(int c = 0; c < 3; c++)
      {
        const float *src = ubase[dy][c] + ko;
        pf[dy][c] = p0 ? __ldg(src) : 0.0f;
        pf1[dy][c] = p1 ? __ldg(src + 1) : 0.0f;
      }
    }
  };
  // the loaded layer as node values (ei + dx, ej + dy)
  auto take_loads = [&](float (&o)[2][2][3])
  {
#pragma unroll
    for(int dy = 0; dy < 2; dy++)
#pragma unroll
      for(int c = 0; c < 3; c++)
      {
        const float v1 = __shfl_down_sync(0xffffffffu, pf[dy][c], 1);
        o[dy][0][c] = pf[dy][c];
        o[dy][1][c] = l == 31 ? pf1[dy][c] : v1;
      }
  };
  const float *Ebase = a.E + e_off;
  float Epf = 0.0f; // modulus of the element layer gathered next
  auto load_E = [&](int e)
  {
    Epf = (e_ok && e >= 0 && e < g.nz) ? __ldg(Ebase + e * eplane) : 0.0f;
  };
  // epilogue inputs of the own node, one node layer ahead
  unsigned fpf = 0;
  float bpf[3] = {0.f, 0.f, 0.f}, ipf[3] = {0.f, 0.f, 0.f}, dpf[3] = {0.f, 0.f, 0.f};
  auto load_out_inputs = [&](int k)
  {
    if(!(own && k >= kb && k < ke))
      return;
    const int n = own_off + k * plane;
    fpf = a.fix[n];
#pragma unroll
    for(int c = 0; c < 3; c++)
    {
      const int id = c * numnp + n;
      if(OP == TC_RESID || OP == TC_CHEB)
        bpf[c] = __ldg(a.b + id);
      if(OP == TC_CHEB)
      {
        ipf[c] = __ldg(a.invd + id);
        dpf[c] = a.c1 != 0.0f ? a.d[id] : 0.0f;
      }
    }
  };

  // Ping-pong register sets, indexed by the parity P of the element layer
  // (counted from the first): cur[P] holds node layer e when element layer
  // e is gathered, which writes node layer e + 1 into cur[P ^ 1]; uq[P] and
  // Eq[P] are the own node value and the element modulus of layer e.
  float cur[2][2][2][3];
  float uq[2][3] = {{0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}};
  float Eq[2] = {0.f, 0.f};
  const int e_first = kb - 1, e_last = ke - 1;
  issue_loads(e_first);
  take_loads(cur[0]);
  issue_loads(e_first + 1);
  load_E(e_first);

  auto gather = [&](auto par, int e)
  {
    constexpr int P = decltype(par)::value;
    take_loads(cur[P ^ 1]);
    issue_loads(e + 2);
    Eq[P] = Epf;
    load_E(e + 1);
    float v[24];
#pragma unroll
    for(int dz = 0; dz < 2; dz++)
#pragma unroll
      for(int dy = 0; dy < 2; dy++)
#pragma unroll
        for(int dx = 0; dx < 2; dx++)
#pragma unroll
          for(int c = 0; c < 3; c++)
            v[3 * local_node(dx, dy, dz) + c] = cur[P ^ dz][dy][dx][c];
#pragma unroll
    for(int c = 0; c < 3; c++)
      uq[P][c] = cur[P][0][0][c];
    // Ke0 annihilates rigid translations, so Ke0 u_e = Ke0 (u_e - t) with t
    // the displacement of local node 0: the BF16 split then rounds strain-size
    // differences instead of displacements (a cantilever tip moves far more
    // than its elements deform).
#pragma unroll
    for(int a_ = 7; a_ >= 0; a_--)
#pragma unroll
      for(int c = 0; c < 3; c++)
        v[3 * a_ + c] -= v[c];
    uint8_t *ah = sm.A[P][mma][0] + cm_off(mrow, 0);
#pragma unroll
    for(int kc = 0; kc < 3; kc++)
    {
      uint32_t hi[4], lo[4];
#pragma unroll
      for(int p = 0; p < 4; p++)
      {
        const float x0 = v[8 * kc + 2 * p], x1 = v[8 * kc + 2 * p + 1];
        hi[p] = bf2_bits(__floats2bfloat162_rn(x0, x1));
        if(TERMS == 3)
        {
          const float h0 = __uint_as_float(hi[p] << 16);
          const float h1 = __uint_as_float(hi[p] & 0xFFFF0000u);
          lo[p] = bf2_bits(__floats2bfloat162_rn(x0 - h0, x1 - h1));
        }
      }
      *reinterpret_cast<uint4 *>(ah + kc * 128) = make_uint4(hi[0], hi[1], hi[2], hi[3]);
      if(TERMS == 3)
        *reinterpret_cast<uint4 *>(ah + kABytes + kc * 128) =
            make_uint4(lo[0], lo[1], lo[2], lo[3]);
    }
  };

  auto issue = [&](int st)
  {
    fence_after();
    const uint32_t bh = saddr(sm.B[0]), bl = saddr(sm.B[1]);
#pragma unroll
    for(int m = 0; m < kMmas; m++)
    {
      const uint32_t d = sm.tmem + (uint32_t)((st * kMmas + m) * 32);
      const uint32_t ah = saddr(sm.A[st][m][0]);
#pragma unroll
      for(int ks = 0; ks < 2; ks++)
      {
        const uint32_t o = (uint32_t)ks * 256u; // two K chunks of 16 B per MMA (K = 16)
        umma(d, smem_desc(ah + o), smem_desc(bh + o), ks);
        if(TERMS == 3)
        {
          umma(d, smem_desc(ah + o), smem_desc(bl + o), 1);
          umma(d, smem_desc(ah + kABytes + o), smem_desc(bh + o), 1);
        }
      }
    }
    umma_commit(saddr(&sm.mbar[st]));
  };

  gather(std::integral_constant<int, 0>{}, e_first);
  load_out_inputs(e_first + 1);
  fence_async_smem();
  fence_before();
  __syncthreads();
  if(t == 0)
    issue(0);

  float carry[3] = {0.0f, 0.0f, 0.0f};
  double dot = 0.0;
  const int nlayers = e_last - e_first + 1;
  int stuck = -1; // iteration whose MMA did not complete in time

  // element layer e = e_first + it, P = it & 1 (also the smem / TMEM stage)
  auto step = [&](auto par, int it) -> bool
  {
    constexpr int P = decltype(par)::value;
    const int e = e_first + it;
    const bool more = it + 1 < nlayers;
    if(more)
    {
      gather(std::integral_constant<int, P ^ 1>{}, e + 1);
      fence_async_smem();
    }
    const bool ok = mbar_wait(saddr(&sm.mbar[P]), (uint32_t)((it >> 1) & 1));
    fence_after();
    float D[24];
    tmem_ld24(sm.tmem + (uint32_t)((P * kMmas + mma) * 32) + ((uint32_t)((w & 3) * 32) << 16),
              D);
    const float Ee = Eq[P];
    // x pairs: node (ei, ej + dy, e + dz) <- element (ei, .) corner dx = 0 and
    // element (ei - 1, .) corner dx = 1 (scaled by the sender's modulus)
    float S[2][2][3];
#pragma unroll
    for(int dz = 0; dz < 2; dz++)
#pragma unroll
      for(int dy = 0; dy < 2; dy++)
#pragma unroll
        for(int c = 0; c < 3; c++)
        {
          const float nb =
              __shfl_up_sync(0xffffffffu, Ee * D[3 * local_node(1, dy, dz) + c], 1);
          S[dy][dz][c] = fmaf(Ee, D[3 * local_node(0, dy, dz) + c], nb);
        }
#pragma unroll
    for(int dz = 0; dz < 2; dz++)
#pragma unroll
      for(int c = 0; c < 3; c++)
        sm.xch[P][dz * 3 + c][w][l] = S[1][dz][c];
    fence_before();
    if(__syncthreads_or(!ok)) // uniform decision of the whole CTA
    {
      stuck = it;
      return false;
    }
    if(more && t == 0)
      issue(P ^ 1);
    // y pairs: node (ei, ej) <- element rows ej (dy = 0) and ej - 1 (dy = 1)
    float T[2][3];
#pragma unroll
    for(int dz = 0; dz < 2; dz++)
#pragma unroll
      for(int c = 0; c < 3; c++)
        T[dz][c] = S[0][dz][c] + (w > 0 ? sm.xch[P][dz * 3 + c][w - 1][l] : 0.0f);
    if(e >= kb && own)
    {
      const int n = own_off + e * plane;
      const unsigned f = fpf;
#pragma unroll
      for(int c = 0; c < 3; c++)
      {
        const int id = c * numnp + n;
        const float ku = carry[c] + T[0][c];
        const bool fixed = (f >> c) & 1u;
        if(OP == TC_APPLY || OP == TC_DOT)
        {
          const float yv = fixed ? 0.0f : ku;
          a.y[id] = yv;
          if(OP == TC_DOT)
            dot += (double)uq[P][c] * (double)yv;
        }
        else if(OP == TC_RESID)
          a.y[id] = fixed ? 0.0f : bpf[c] - ku;
        else
        {
          const float dn = fixed ? 0.0f : fmaf(a.c1, dpf[c], a.c2 * ipf[c] * (bpf[c] - ku));
          a.d[id] = dn;
          a.y[id] = uq[P][c] + dn;
        }
      }
    }
    load_out_inputs(e + 1);
#pragma unroll
    for(int c = 0; c < 3; c++)
      carry[c] = T[1][c];
    return true;
  };
  for(int it = 0; it < nlayers; it += 2)
  {
    if(!step(std::integral_constant<int, 0>{}, it))
      break;
    if(it + 1 < nlayers && !step(std::integral_constant<int, 1>{}, it + 1))
      break;
  }
  if(stuck >= 0)
  {
    // give the MMA in flight a bounded second chance to land before freeing TMEM
    mbar_wait(saddr(&sm.mbar[stuck & 1]), (uint32_t)((stuck >> 1) & 1));
    if(t == 0)
      atomicExch(a.err, 1);
  }
  fence_before();
  __syncthreads();
  if(w == 0)
  {
    fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(sm.tmem),
                 "r"(kTmemCols));
  }
  if(OP == TC_DOT)
  {
    double v[1] = {dot};
    block_sum<1>(v, sm.red);
    const int nblk = gridDim.x * gridDim.y;
    const int bid = blockIdx.y * gridDim.x + blockIdx.x;
    if(t == 0)
      a.partials[bid] = v[0];
    __shared__ bool last;
    __threadfence();
    __syncthreads();
    if(t == 0)
      last = atomicAdd(&a.s->counter, 1u) == (unsigned)(nblk - 1);
    __syncthreads();
    if(last)
    {
      __threadfence();
      double r[1];
      sum_partials<1>(a.partials, nblk, r, sm.red);
      if(t == 0)
      {
        a.s->pAp = r[0];
        a.s->alpha = a.s->zr / r[0];
        a.s->counter = 0;
      }
    }
  }
}

// ---------------------------------------------------------------- host side
template <int TERMS> static size_t tc_smem_bytes() { return sizeof(tc::Smem<TERMS>) + 128; }

template <int OP, int TERMS> static int tc_prepare()
{
  static int occ_of[kMaxDevices] = {};
  int &occ = occ_of[device_slot()];
  if(!occ)
  {
    ICK(cudaFuncSetAttribute(k_ku_tc<OP, TERMS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)tc_smem_bytes<TERMS>()));
    int o = 0;
    ICK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, k_ku_tc<OP, TERMS>, tc::kThreads,
                                                      tc_smem_bytes<TERMS>()));
    occ = o < 1 ? 1 : o;
  }
  return occ;
}

// Node layers per CTA: few enough that every SM slot gets work, many enough
// that the one-layer z halo stays cheap; among those, the count whose last
// wave is fullest.
int pick_layers(long tiles, int NZ, long slots, long max_ctas)
{
  int best = NZ;
  double best_eff = -1.0;
  for(int kc = 8; kc <= NZ + 7; kc++)
  {
    const long z = (NZ + kc - 1) / kc;
    const long ctas = tiles * z;
    if(ctas > max_ctas)
      continue;
    const double waves = (double)ctas / slots;
    const double fill = waves / std::ceil(waves);
    const double eff = fill * (double)kc / (kc + 1);
    if(eff > best_eff + 1e-9)
    {
      best_eff = eff;
      best = kc;
    }
    if(z == 1)
      break;
  }
  return best;
}

void launch_ku_tc(icarat_ctx *c, int op, int terms, TcArgs a, cudaStream_t st)
{
  const GridDev &g = a.g;
  IREQUIRE(3L * g.numnp < (1L << 31), ICARAT_ERR_UNSUPPORTED,
           "grid too large for 32-bit offsets");
  a.keb = c->d_keb;
  a.err = c->d_tc_err;
  a.tiles_x = (g.NX + tc::kOX - 1) / tc::kOX;
  const int tiles_y = (g.NY + tc::kOY - 1) / tc::kOY;
  const long txy = (long)a.tiles_x * tiles_y;
  IREQUIRE(op != TC_DOT || txy <= kMaxRedBlocks, ICARAT_ERR_UNSUPPORTED,
           "grid too wide for the tensor-core reduction");
#define ICARAT_TC_CASE(O, T)                                                      \
  if(op == O && terms == T)                                                     \
  {                                                                             \
    const int occ = tc_prepare<O, T>();                                         \
    a.kc = pick_layers(txy, g.NZ, (long)c->sm_count * occ,                      \
                       O == TC_DOT ? (long)kMaxRedBlocks : (1L << 30));         \
    const dim3 grid((unsigned)txy, (unsigned)((g.NZ + a.kc - 1) / a.kc));       \
    note_launch();                                                              \
    launch_chained(k_ku_tc<O, T>, grid, tc::kThreads, tc_smem_bytes<T>(), st, a); \
    ICK(cudaGetLastError());                                                    \
    return;                                                                     \
  }
  ICARAT_TC_CASE(TC_APPLY, 1)
  ICARAT_TC_CASE(TC_APPLY, 3)
  ICARAT_TC_CASE(TC_RESID, 1)
  ICARAT_TC_CASE(TC_RESID, 3)
  ICARAT_TC_CASE(TC_CHEB, 1)
  ICARAT_TC_CASE(TC_CHEB, 3)
  ICARAT_TC_CASE(TC_DOT, 1)
  ICARAT_TC_CASE(TC_DOT, 3)
#undef ICARAT_TC_CASE
  throw Error{ICARAT_ERR_ARG, "unknown tensor-core operator variant"};
}

} // namespace icarat_b200
