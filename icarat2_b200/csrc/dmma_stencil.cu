// Element-by-element FP64 K u on the FP64 tensor cores (mma.sync m8n8k4 f64,
// the DMMA path of sm_100a; tcgen05 has no FP64 kind).  No reference
// counterpart: the reference assembles K and multiplies in FP64 on the CPU.
//
// For a group of 8 elements the element products form one GEMM
//     D (8 x 24) = U (8 x 24) Ke0^T (24 x 24),
// row e of U = the 24 nodal displacements of element e (DOF 3 a + c, local
// node a, component c).  One m8n8k4 MMA multiplies an 8 x 4 slice of U by a
// 4 x 8 slice of Ke0^T, so a group takes 6 (K) x 3 (N) MMAs; the 18 Ke0^T
// fragments stay in registers for the whole launch.  The products are exact
// FP64 FMAs; the result differs from the node stencil only in the order of
// the sums.  The moduli E_e scale the rows of D afterwards.
//
// Tile and sweep as the tcgen05 operator (tc_stencil.cu): a CTA of 8 warps
// owns a column of 31 x 7 nodes (x, y) over a range of node layers (z).  Per
// element layer warp w multiplies the 32 elements of element row j0 - 1 + w
// (4 groups of 8), so every owned node has all 4 elements of the layer
// inside the tile; the one-element halo is recomputed by the neighbouring
// CTA.  Node sums need no atomics: x pairs by a warp shuffle, y pairs
// through shared memory and z pairs in registers carried to the next layer.
//
// Fragment layout (A row-major, B column-major): lane l = 4 r + q holds
// U[element r][DOF 4 kc + q] of its group, Ke0[8 nc + r][4 kc + q] and
// D[element r][rows 8 nc + 2 q, 8 nc + 2 q + 1].  A lane therefore gathers
// DOFs q, q + 4, ..., q + 20 of elements r, r + 8, r + 16, r + 24 of the
// warp's row.  DOF d + 12 of an element is DOF d of the element one layer up
// (12 = 4 corner nodes x 3 components, with the same in-plane corner and
// component), so the upper half gathered for element layer e is the lower
// half of layer e + 1 and stays in registers: each lane loads 12 values per
// layer, issued one layer ahead of their use.  D passes through shared
// memory (row-major by D row, 36 doubles per row: conflict-free fragment
// writes and element-per-lane reads) to the element-per-lane order of the
// node sums.
#include <algorithm>

#include "stencil.cuh"

namespace icarat_b200
{
namespace dm
{

constexpr int kTX = 32, kTY = 8;            // elements per tile row / rows
constexpr int kOX = kTX - 1, kOY = kTY - 1; // owned nodes per layer (x, y)
constexpr int kThreads = kTX * kTY;
constexpr int kPitch = 36;                  // doubles per D row in shared memory

struct Smem
{
  double D[kTY][24][kPitch];  // [warp][D row][element]
  double xch[2][6][kTY][32];  // [stage][dz * 3 + c][warp][lane]
  double kf[6][3][32];        // Ke0^T fragments [K chunk][N chunk][lane]
  double red[32];
};

__device__ __forceinline__ void dmma(double (&d)[2], double a, double b)
{
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, "
               "{%0,%1};\n"
               : "+d"(d[0]), "+d"(d[1])
               : "d"(a), "d"(b));
}

// m16n8k8 (sm_90+): rows g and g + 8 of A / D are the two 8-element groups
// of a pair, so with g = lane / 4, t = lane % 4 the fragments are those of
// two m8n8k4 groups and two K chunks: a = {U0[k0], U1[k0], U0[k1], U1[k1]},
// b = {K[k0], K[k1]}, d = {D0[0..1], D1[0..1]}
__device__ __forceinline__ void dmma16(double (&d0)[2], double (&d1)[2], double a0, double a1,
                                       double a2, double a3, double b0, double b1)
{
  asm volatile("mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, "
               "{%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
               : "+d"(d0[0]), "+d"(d0[1]), "+d"(d1[0]), "+d"(d1[1])
               : "d"(a0), "d"(a1), "d"(a2), "d"(a3), "d"(b0), "d"(b1));
}

} // namespace dm

// Work: the (tile, node layer) pairs in tile-major order, split evenly over
// the CTAs (two per SM); a CTA runs its range as one or two tile segments,
// each with one element layer of z halo.  The Ke0^T fragments live in shared
// memory so that a thread fits in 128 registers: two CTAs per SM, whose
// layers drift apart, keep the tensor pipe busy while the other one sums.
template <int OP>
__global__ void __launch_bounds__(dm::kThreads, 2) k_ku_dmma(DmArgs a)
{
  using namespace dm;
  extern __shared__ __align__(16) uint8_t dm_smem_raw[];
  Smem &sm = *reinterpret_cast<Smem *>(dm_smem_raw);
  if(halted(a.halt) || (OP == TC_DOT && a.s->done))
    return;
  const int t = threadIdx.x, w = t >> 5, l = t & 31;
  const int q = l & 3, r = l >> 2;
  const GridDev g = a.g;
  const int plane = g.NX * g.NY, eplane = g.nx * g.ny, numnp = g.numnp;

  // Ke0^T fragments: kf[kc][nc][lane] = Ke0[8 nc + r][4 kc + q]
  for(int i = t; i < 6 * 3 * 32; i += kThreads)
  {
    const int kc = i / 96, nc = (i / 32) % 3, ln = i % 32;
    sm.kf[kc][nc][ln] = a.ke.k[(8 * nc + (ln >> 2)) * 24 + 4 * kc + (ln & 3)];
  }
  __syncthreads();

  double dot = 0.0;
  const long work = (long)a.tiles * g.NZ;
  const long w_begin = work * blockIdx.x / gridDim.x;
  const long w_end = work * (blockIdx.x + 1) / gridDim.x;
  for(long wpos = w_begin; wpos < w_end;)
  {
    const int tile = (int)(wpos / g.NZ);
    const int kb = (int)(wpos % g.NZ);
    const int ke = (int)min((long)g.NZ, kb + (w_end - wpos));
    wpos += ke - kb;
    const int i0 = (tile % a.tiles_x) * kOX, j0 = (tile / a.tiles_x) * kOY;
    const int ej = j0 - 1 + w;
    // the element of this lane in the node sums (x = lane, y = warp) and the
    // node it owns
    const int ei = i0 - 1 + l;
    const bool e_ok = ei >= 0 && ei < g.nx && ej >= 0 && ej < g.ny;
    const int e_off = ei + ej * g.nx;
    const bool own = l >= 1 && w >= 1 && ei < g.NX && ej < g.NY;
    const int own_off = ei + ej * g.NX;
    // groups of 8 elements with at least one element inside the grid (warp
    // uniform); the others skip their MMAs and contribute zeros
    bool grp_ok[4];
#pragma unroll
    for(int gg = 0; gg < 4; gg++)
    {
      const int x0 = i0 - 1 + 8 * gg;
      grp_ok[gg] = ej >= 0 && ej < g.ny && x0 + 7 >= 0 && x0 < g.nx;
    }

    // gather of slot h = DOF 12 + 4 h + q (upper corner) and DOF 4 h + q (the
    // same in-plane corner one layer down) of group gg: node x = gx0[h] + 8 gg
    // on node row gy[h]; offsets are rebuilt per load to save registers
    int gx0[3], gbase[3];
    unsigned gymask = 0; // bit h: node row inside the grid
#pragma unroll
    for(int h = 0; h < 3; h++)
    {
      const int d = 12 + 4 * h + q;
      const int corner = d / 3 - 4, comp = d % 3;
      const int ax = (corner == 1 || corner == 2) ? 1 : 0, ay = corner >= 2 ? 1 : 0;
      gx0[h] = i0 - 1 + r + ax;
      const int y = ej + ay;
      if(y >= 0 && y < g.NY)
        gymask |= 1u << h;
      gbase[h] = comp * numnp + y * g.NX;
    }
    auto load_layer = [&](int k, double (&o)[4][3])
    {
      const bool kin = k >= 0 && k < g.NZ;
      const int ko = kin ? k * plane : 0;
#pragma unroll
      for(int gg = 0; gg < 4; gg++)
#pragma unroll
        for(int h = 0; h < 3; h++)
        {
          const int x = gx0[h] + 8 * gg;
          const bool ok = kin && ((gymask >> h) & 1u) && x >= 0 && x < g.NX;
          o[gg][h] = ok ? __ldg(a.u + (gbase[h] + x + ko)) : 0.0;
        }
    };
    const double *Ebase = a.E + e_off;
    auto load_E = [&](int e) -> double
    { return (e_ok && e >= 0 && e < g.nz) ? __ldg(Ebase + e * eplane) : 0.0; };
    // epilogue inputs of the own node, one node layer ahead
    unsigned fpf = 0;
    double upf[3] = {0.0, 0.0, 0.0}, bpf[3] = {0.0, 0.0, 0.0}, ipf[3] = {0.0, 0.0, 0.0},
           dpf[3] = {0.0, 0.0, 0.0};
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
        if(OP == TC_DOT || OP == TC_CHEB)
          upf[c] = __ldg(a.u + id);
        if(OP == TC_RESID || OP == TC_CHEB)
          bpf[c] = __ldg(a.b + id);
        if(OP == TC_CHEB)
        {
          ipf[c] = __ldg(a.invd + id);
          dpf[c] = a.c1 != 0.0 ? a.d[id] : 0.0;
        }
      }
    };

    // element products of the layer whose lower / upper node values are in
    // lo / up: issued into acc (the tensor pipe works on them meanwhile),
    // stored to D[stage] later
    // element products of the layer whose lower / upper node values are in
    // lo / up, one pair of groups (M = 16 for m16n8k8, K chunk pairs as
    // K = 8) at a time, straight into D; groups outside the grid (warp
    // uniform) skip their MMAs and store zeros
    auto mma_layer = [&](const double (&lo)[4][3], const double (&up)[4][3])
    {
#pragma unroll
      for(int pr = 0; pr < 2; pr++)
      {
        const int g0 = 2 * pr, g1 = 2 * pr + 1;
        double acc[2][3][2];
#pragma unroll
        for(int m = 0; m < 2; m++)
#pragma unroll
          for(int nc = 0; nc < 3; nc++)
            acc[m][nc][0] = acc[m][nc][1] = 0.0;
        if(grp_ok[g0] && grp_ok[g1])
        {
#pragma unroll
          for(int k2 = 0; k2 < 3; k2++)
#pragma unroll
            for(int nc = 0; nc < 3; nc++)
            {
              const int ka = 2 * k2, kb_ = 2 * k2 + 1;
              dmma16(acc[0][nc], acc[1][nc], ka < 3 ? lo[g0][ka] : up[g0][ka - 3],
                     ka < 3 ? lo[g1][ka] : up[g1][ka - 3],
                     kb_ < 3 ? lo[g0][kb_] : up[g0][kb_ - 3],
                     kb_ < 3 ? lo[g1][kb_] : up[g1][kb_ - 3], sm.kf[ka][nc][l],
                     sm.kf[kb_][nc][l]);
            }
        }
        else
        {
#pragma unroll
          for(int m = 0; m < 2; m++)
            if(grp_ok[g0 + m])
#pragma unroll
              for(int kc = 0; kc < 6; kc++)
#pragma unroll
                for(int nc = 0; nc < 3; nc++)
                  dmma(acc[m][nc], kc < 3 ? lo[g0 + m][kc] : up[g0 + m][kc - 3],
                       sm.kf[kc][nc][l]);
        }
#pragma unroll
        for(int m = 0; m < 2; m++)
#pragma unroll
          for(int nc = 0; nc < 3; nc++)
#pragma unroll
            for(int s_ = 0; s_ < 2; s_++)
              sm.D[w][8 * nc + 2 * q + s_][8 * (g0 + m) + r] = acc[m][nc][s_];
      }
    };

    const int e_first = kb - 1, e_last = ke - 1;
    double lo[4][3], up[4][3];
    load_layer(e_first, lo);
    load_layer(e_first + 1, up);
    double Ecur = load_E(e_first), Enext = load_E(e_first + 1);
    load_out_inputs(kb);
    double carry[3] = {0.0, 0.0, 0.0};

    // element layer e = e_first + it, stage P = it & 1
    auto step = [&](auto par, int it)
    {
      constexpr int P = decltype(par)::value;
      const int e = e_first + it;
      mma_layer(lo, up); // node layers e, e + 1
#pragma unroll
      for(int gg = 0; gg < 4; gg++)
#pragma unroll
        for(int h = 0; h < 3; h++)
          lo[gg][h] = up[gg][h];
      if(e < e_last)
        load_layer(e + 2, up);
      const double Ee = Ecur;
      Ecur = Enext;
      Enext = load_E(e + 2);
      __syncwarp();
      // x pairs: node (ei, ej + dy, e + dz) <- element (ei, .) corner dx = 0
      // and element (ei - 1, .) corner dx = 1 (scaled by the sender's modulus)
      double S[2][2][3];
#pragma unroll
      for(int dz = 0; dz < 2; dz++)
#pragma unroll
        for(int dy = 0; dy < 2; dy++)
#pragma unroll
          for(int c = 0; c < 3; c++)
          {
            const double d1 = sm.D[w][3 * local_node(1, dy, dz) + c][l];
            const double d0 = sm.D[w][3 * local_node(0, dy, dz) + c][l];
            const double nb = __shfl_up_sync(0xffffffffu, Ee * d1, 1);
            S[dy][dz][c] = fma(Ee, d0, nb);
          }
#pragma unroll
      for(int dz = 0; dz < 2; dz++)
#pragma unroll
        for(int c = 0; c < 3; c++)
          sm.xch[P][dz * 3 + c][w][l] = S[1][dz][c];
      __syncthreads();
      // y pairs: node (ei, ej) <- element rows ej (dy = 0) and ej - 1 (dy = 1)
      double T[2][3];
#pragma unroll
      for(int dz = 0; dz < 2; dz++)
#pragma unroll
        for(int c = 0; c < 3; c++)
          T[dz][c] = S[0][dz][c] + (w > 0 ? sm.xch[P][dz * 3 + c][w - 1][l] : 0.0);
      if(e >= kb && own)
      {
        const int n = own_off + e * plane;
        const unsigned f = fpf;
#pragma unroll
        for(int c = 0; c < 3; c++)
        {
          const int id = c * numnp + n;
          const double ku = carry[c] + T[0][c];
          const bool fixed = (f >> c) & 1u;
          if(OP == TC_APPLY || OP == TC_DOT)
          {
            const double yv = fixed ? 0.0 : ku;
            a.y[id] = yv;
            if(OP == TC_DOT)
              dot += upf[c] * yv;
          }
          else if(OP == TC_RESID)
            a.y[id] = fixed ? 0.0 : bpf[c] - ku;
          else
          {
            const double dn = fixed ? 0.0
                                    : (a.c1 != 0.0 ? a.c1 * dpf[c] : 0.0) +
                                          a.c2 * ipf[c] * (bpf[c] - ku);
            a.d[id] = dn;
            a.y[id] = upf[c] + dn;
          }
        }
      }
      load_out_inputs(e + 1);
#pragma unroll
      for(int c = 0; c < 3; c++)
        carry[c] = T[1][c];
    };
    const int nlayers = e_last - e_first + 1;
    for(int it = 0; it < nlayers; it += 2)
    {
      step(std::integral_constant<int, 0>{}, it);
      if(it + 1 < nlayers)
        step(std::integral_constant<int, 1>{}, it + 1);
    }
    __syncthreads(); // the next segment reuses the stages
  }

  if(OP == TC_DOT)
  {
    double v[1] = {dot};
    block_sum<1>(v, sm.red);
    if(t == 0)
      a.partials[blockIdx.x] = v[0];
    if(last_block(&a.s->counter))
    {
      double s[1];
      sum_partials<1>(a.partials, gridDim.x, s, sm.red);
      if(t == 0)
      {
        a.s->pAp = s[0];
        a.s->alpha = a.s->zr / s[0];
        a.s->counter = 0;
      }
    }
  }
}

// ---------------------------------------------------------------- host side
template <int OP> static int dm_prepare()
{
  static int occ_of[kMaxDevices] = {};
  int &occ = occ_of[device_slot()];
  if(!occ)
  {
    ICK(cudaFuncSetAttribute(k_ku_dmma<OP>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)sizeof(dm::Smem)));
    int o = 0;
    ICK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, k_ku_dmma<OP>, dm::kThreads,
                                                      sizeof(dm::Smem)));
    occ = o < 1 ? 1 : o;
  }
  return occ;
}

bool dmma_fits(const GridDev &g)
{
  const long tiles = (long)((g.NX + dm::kOX - 1) / dm::kOX) * ((g.NY + dm::kOY - 1) / dm::kOY);
  return 3L * g.numnp < (1L << 31) && tiles <= kMaxRedBlocks;
}

void launch_ku_dmma(icarat_ctx *c, int op, DmArgs a, cudaStream_t st)
{
  const GridDev &g = a.g;
  IREQUIRE(dmma_fits(g), ICARAT_ERR_UNSUPPORTED,
           "grid too large for the FP64 tensor-core operator");
  a.ke = c->ke0;
  a.tiles_x = (g.NX + dm::kOX - 1) / dm::kOX;
  a.tiles = a.tiles_x * ((g.NY + dm::kOY - 1) / dm::kOY);
  // one CTA per SM slot, at least 8 node layers of work each
  const long work = (long)a.tiles * g.NZ;
#define ICARAT_DM_CASE(O)                                                         \
  if(op == O)                                                                     \
  {                                                                               \
    const int occ = dm_prepare<O>();                                              \
    long grid = std::min((long)c->sm_count * occ, std::max(1L, work / 8));        \
    grid = std::min(grid, (long)kMaxRedBlocks);                                   \
    note_launch();                                                                \
    k_ku_dmma<O><<<(unsigned)grid, dm::kThreads, sizeof(dm::Smem), st>>>(a);      \
    ICK(cudaGetLastError());                                                      \
    return;                                                                       \
  }
  ICARAT_DM_CASE(TC_APPLY)
  ICARAT_DM_CASE(TC_RESID)
  ICARAT_DM_CASE(TC_CHEB)
  ICARAT_DM_CASE(TC_DOT)
#undef ICARAT_DM_CASE
  throw Error{ICARAT_ERR_ARG, "unknown FP64 tensor-core operator variant"};
}

} // namespace icarat_b200
