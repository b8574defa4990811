// 3x3x3 convolution of the learned preconditioner's U-net on the
// 5th-generation tensor cores (tcgen05, BF16 operands, FP32 accumulation in
// TMEM): the forward pass of every conv3 layer, bias and ReLU fused, BF16
// out.  No reference counterpart (the reference has no learned part).
//
// Implicit GEMM per CTA: D (128 voxels x C_out) += A_tap (128 x 16 input
// channels) B_tap^T (16 x C_out) over the 27 taps and the 16-channel chunks
// of C_in.  The 128 output voxels of one MMA are an 8 (x) x 16 (y) patch of
// one z-plane; a CTA owns ZT = 4 consecutive z-planes of the patch (four
// accumulators in TMEM) so that the staged weights and the staged input
// planes serve four MMAs each.
//
// Operands in shared memory, K-major without swizzle (core matrices of 8
// rows x 16 bytes):
//   input  [ci half h (8 channels)][plane p][row (yy * 10 + xx)][8 ch] for
//          the patch with a one-voxel halo: xx, yy, p cover x0-1..x0+8,
//          y0-1..y0+16, z0-1..z0+ZT; outside the grid the values are 0 (the
//          convolution's zero padding).  An 8-voxel x-row of the patch is one
//          core-matrix group, the groups (y) are 160 bytes apart, so the
//          shifted view of tap (dx, dy, dz) is a descriptor whose start moves
//          by (dz planes, (1 + dy) 10 + (1 + dx) rows): no im2col.
//   weights[tap][h][co][8 ch], packed once per weight update (k_conv_pack).
// One thread issues the 27 x ZT MMAs of a chunk and commits them to an
// mbarrier; the CTA waits (bounded) before staging the next chunk.  The
// epilogue reads each accumulator with tcgen05.ld (thread = TMEM lane =
// voxel), adds the bias, applies the ReLU and stores BF16 channel-major.
#include <cuda_bf16.h>

#include <algorithm>

#include "internal.cuh"

namespace icarat_b200
{
namespace ctc
{

constexpr int kThreads = 128;
constexpr int kPX = 8, kPY = 16;                    // output patch (x, y) per MMA
constexpr int kZT = 4;                              // z-planes per CTA
constexpr int kRows = (kPX + 2) * (kPY + 2);        // staged rows per plane (with halo)
constexpr int kPlanes = kZT + 2;
constexpr uint32_t kActHalf = kPlanes * kRows * 16; // bytes of one 8-channel half
constexpr long kWaitLimit = 1L << 24;               // mbarrier polls before giving up

__device__ __forceinline__ uint32_t saddr(const void *p)
{
  return (uint32_t)__cvta_generic_to_shared(p);
}

// K-major, no swizzle: start, K-chunk stride (LBO), 8-row group stride (SBO)
__device__ __forceinline__ uint64_t desc(uint32_t addr, uint32_t lbo, uint32_t sbo)
{
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// kind::f16 instruction descriptor: D F32, A and B BF16, both K-major, M = 128
__device__ __forceinline__ uint32_t idesc(int n)
{
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) |
         ((uint32_t)(128 >> 4) << 24);
}

__device__ __forceinline__ void umma(uint32_t d, uint64_t a, uint64_t b, uint32_t id, int acc)
{
  asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
               "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d),
               "l"(a), "l"(b), "r"(id), "r"(acc));
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

} // namespace ctc

// wpk[chunk][tap][h][co][j] = W[co][16 chunk + 8 h + j][tap] (0 past cin)
__global__ void k_conv_pack(const __nv_bfloat16 *__restrict__ W, int cin, int cout,
                            __nv_bfloat16 *__restrict__ wpk)
{
  const int nchunk = (cin + 15) / 16;
  const long n = (long)nchunk * 27 * 2 * cout * 8;
  for(long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
      i += (long)gridDim.x * blockDim.x)
  {
    const int j = (int)(i % 8), co = (int)((i / 8) % cout), h = (int)((i / (8L * cout)) % 2);
    const int tap = (int)((i / (16L * cout)) % 27), ch = (int)(i / (16L * cout * 27));
    const int ci = 16 * ch + 8 * h + j;
    wpk[i] = ci < cin ? W[((long)co * cin + ci) * 27 + tap] : __float2bfloat16_rn(0.0f);
  }
}

__global__ void __launch_bounds__(ctc::kThreads)
    k_conv3_tc(int X, int Y, int Z, long V, const __nv_bfloat16 *__restrict__ x, int cin,
               const __nv_bfloat16 *__restrict__ wpk, const float *__restrict__ bias, int cout,
               __nv_bfloat16 *__restrict__ y, int tmem_cols, int *err)
{
  using namespace ctc;
  extern __shared__ __align__(128) uint8_t conv_smem_raw[];
  uint8_t *act = conv_smem_raw;                // 2 halves x kActHalf
  uint8_t *wsm = conv_smem_raw + 2 * kActHalf; // 27 x 2 x cout x 16 B
  __shared__ __align__(8) unsigned long long mbar;
  __shared__ uint32_t tmem_base;
  const int t = threadIdx.x, w = t >> 5;
  const int tiles_x = (X + kPX - 1) / kPX, tiles_y = (Y + kPY - 1) / kPY;
  const int tx = blockIdx.x % tiles_x, ty = (blockIdx.x / tiles_x) % tiles_y;
  const int tz = blockIdx.x / (tiles_x * tiles_y);
  const int x0 = tx * kPX, y0 = ty * kPY, z0 = tz * kZT;
  const long plane = (long)X * Y;
  if(t == 0)
  {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(saddr(&mbar)), "r"(1));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if(w == 0)
  {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     saddr(&tmem_base)),
                 "r"(tmem_cols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_base;

  const int nchunk = (cin + 15) / 16;
  const uint32_t wbytes = 27u * 2u * (uint32_t)cout * 16u;
  const uint32_t id = idesc(cout);
  bool ok = true;
  for(int ch = 0; ch < nchunk && ok; ch++)
  {
    // ---- stage the input patch of channels 16 ch .. 16 ch + 15
    for(int item = t; item < 2 * kPlanes * kRows; item += kThreads)
    {
      const int h = item / (kPlanes * kRows);
      const int p = (item / kRows) % kPlanes, row = item % kRows;
      const int xx = x0 - 1 + row % (kPX + 2), yy = y0 - 1 + row / (kPX + 2), zz = z0 - 1 + p;
      const bool in = xx >= 0 && xx < X && yy >= 0 && yy < Y && zz >= 0 && zz < Z;
      const long v = in ? xx + yy * (long)X + zz * plane : 0;
      uint32_t packed[4];
#pragma unroll
      for(int j = 0; j < 8; j += 2)
      {
        const int c0 = 16 * ch + 8 * h + j;
        const unsigned short lo =
            (in && c0 < cin) ? __bfloat16_as_ushort(x[(long)c0 * V + v]) : (unsigned short)0;
        const unsigned short hi =
            (in && c0 + 1 < cin) ? __bfloat16_as_ushort(x[(long)(c0 + 1) * V + v])
                                 : (unsigned short)0;
        packed[j / 2] = (uint32_t)lo | ((uint32_t)hi << 16);
      }
      *reinterpret_cast<uint4 *>(act + h * kActHalf + (p * kRows + row) * 16) =
          make_uint4(packed[0], packed[1], packed[2], packed[3]);
    }
    // ---- stage the packed weights of the chunk
    const uint4 *wsrc = reinterpret_cast<const uint4 *>(wpk + (long)ch * 27 * 2 * cout * 8);
    for(uint32_t q = t; q < wbytes / 16; q += kThreads)
      reinterpret_cast<uint4 *>(wsm)[q] = __ldg(wsrc + q);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if(t == 0)
    {
      const uint32_t abase = saddr(act), bbase = saddr(wsm);
      for(int zt = 0; zt < kZT; zt++)
        for(int tap = 0; tap < 27; tap++)
        {
          const int dx = tap % 3, dy = (tap / 3) % 3, dz = tap / 9; // offsets + 1
          const uint32_t arow = (uint32_t)((zt + dz) * kRows + dy * (kPX + 2) + dx);
          const uint64_t a = desc(abase + arow * 16u, kActHalf, (kPX + 2) * 16);
          const uint64_t b = desc(bbase + (uint32_t)tap * 2u * cout * 16u, (uint32_t)cout * 16u,
                                  128u);
          umma(tmem + (uint32_t)(zt * cout), a, b, id, (ch > 0 || tap > 0) ? 1 : 0);
        }
      asm volatile(
          "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
              saddr(&mbar))
          : "memory");
    }
    // the stage is reused by the next chunk, and TMEM is read after the last
    ok = mbar_wait(saddr(&mbar), (uint32_t)(ch & 1));
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    ok = __syncthreads_and(ok);
  }
  if(!ok)
  {
    // give the MMAs in flight a bounded second chance to land before TMEM
    // is freed, and report
    mbar_wait(saddr(&mbar), (uint32_t)((nchunk - 1) & 1));
    if(t == 0)
      atomicExch(err, 1);
  }
  else
  {
    // ---- epilogue: thread t = TMEM lane t = voxel (x0 + t % 8, y0 + t / 8)
    const int vx = x0 + t % kPX, vy = y0 + t / kPX;
    for(int zt = 0; zt < kZT; zt++)
    {
      const int vz = z0 + zt;
      const bool valid = vx < X && vy < Y && vz < Z;
      const long v = vx + vy * (long)X + vz * plane;
      for(int c0 = 0; c0 < cout; c0 += 16)
      {
        uint32_t r[16];
        const uint32_t taddr = tmem + ((uint32_t)(w * 32) << 16) + (uint32_t)(zt * cout + c0);
        asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, "
                     "%7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
                     : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
                       "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]),
                       "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
                     : "r"(taddr));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        if(valid)
#pragma unroll
          for(int q = 0; q < 16; q++)
          {
            const float o = fmaxf(__uint_as_float(r[q]) + bias[c0 + q], 0.0f);
            y[(long)(c0 + q) * V + v] = __float2bfloat16_rn(o);
          }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if(w == 0)
  {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(tmem_cols));
  }
}

long conv3_tc_packed_size(int cin, int cout)
{
  return (long)((cin + 15) / 16) * 27 * 2 * cout * 8;
}

void conv3_tc_pack(const uint16_t *W, int cin, int cout, uint16_t *wpk, cudaStream_t st)
{
  const long n = conv3_tc_packed_size(cin, cout);
  note_launch();
  k_conv_pack<<<(unsigned)std::min(4096L, (n + 255) / 256), 256, 0, st>>>(
      reinterpret_cast<const __nv_bfloat16 *>(W), cin, cout,
      reinterpret_cast<__nv_bfloat16 *>(wpk));
  ICK(cudaGetLastError());
}

void conv3_tc_fwd(int X, int Y, int Z, long V, const uint16_t *x, int cin, const uint16_t *wpk,
                  const float *bias, int cout, uint16_t *y, int *err, cudaStream_t st)
{
  IREQUIRE(cout % 16 == 0 && cout >= 16 && cout <= 128, ICARAT_ERR_ARG,
           "tensor-core convolution needs 16..128 output channels in steps of 16");
  constexpr size_t kMaxSmem = 2 * ctc::kActHalf + 27 * 2 * 128 * 16;
  static bool configured[kMaxDevices] = {};
  bool &done = configured[device_slot()];
  if(!done)
  {
    ICK(cudaFuncSetAttribute(k_conv3_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)kMaxSmem));
    done = true;
  }
  const size_t smem = 2 * ctc::kActHalf + 27u * 2u * (size_t)cout * 16u;
  int cols = 32;
  while(cols < ctc::kZT * cout)
    cols *= 2;
  const long tiles = (long)((X + ctc::kPX - 1) / ctc::kPX) * ((Y + ctc::kPY - 1) / ctc::kPY) *
                     ((Z + ctc::kZT - 1) / ctc::kZT);
  note_launch();
  k_conv3_tc<<<(unsigned)tiles, ctc::kThreads, smem, st>>>(
      X, Y, Z, V, reinterpret_cast<const __nv_bfloat16 *>(x), cin,
      reinterpret_cast<const __nv_bfloat16 *>(wpk), bias, cout,
      reinterpret_cast<__nv_bfloat16 *>(y), cols, err);
  ICK(cudaGetLastError());
}

} // namespace icarat_b200
