// Context setup: structured hexa8 box, Dirichlet boxes, DOF numbering, point
// loads, device arrays, and the numeq <-> node-vector conversions.
#include <climits>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>

#include "internal.cuh"

namespace icarat_b200
{

double *dalloc(size_t n)
{
  void *p = nullptr;
  if(n == 0)
    n = 1;
  cudaError_t e = cudaMalloc(&p, n * sizeof(double));
  if(e != cudaSuccess)
    throw Error{ICARAT_ERR_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e)};
  return static_cast<double *>(p);
}

void dfree(void *p)
{
  if(p)
    cudaFree(p);
}

// numeq vector -> node vector (constrained components 0)
__global__ void k_scatter_free(int numeq, const int *__restrict__ free_idx,
                               const double *__restrict__ in,
                               double *__restrict__ out)
{
  for(int r = blockIdx.x * blockDim.x + threadIdx.x; r < numeq;
      r += gridDim.x * blockDim.x)
    out[free_idx[r]] = in[r];
}

__global__ void k_gather_free(int numeq, const int *__restrict__ free_idx,
                              const double *__restrict__ in,
                              double *__restrict__ out)
{
  for(int r = blockIdx.x * blockDim.x + threadIdx.x; r < numeq;
      r += gridDim.x * blockDim.x)
    out[r] = in[free_idx[r]];
}

// SIMP (src/problem/elasticity.hpp:13-17)
// (E32: the same moduli rounded to FP32 for the reduced-precision operators;
// elements removed by a selection have no stiffness at all: E = 0)
__global__ void k_simp(int n, const double *__restrict__ rho, double e1,
                       double e2, double p, const uint8_t *__restrict__ emask,
                       double *__restrict__ E, float *__restrict__ E32)
{
  for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
      i += gridDim.x * blockDim.x)
  {
    double rp = pow(rho[i], p);
    double e = (1.0 - rp) * e1 + rp * e2;
    if(emask && !emask[i])
      e = 0.0;
    E[i] = e;
    E32[i] = (float)e;
  }
}

// kept -> box element layout (removed elements 0 beforehand) and back
__global__ void k_sel_scatter(int n, const int *__restrict__ map,
                              const double *__restrict__ in, double *__restrict__ out)
{
  for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
      i += gridDim.x * blockDim.x)
    out[map[i]] = in[i];
}

__global__ void k_sel_gather(int n, const int *__restrict__ map,
                             const double *__restrict__ in, double *__restrict__ out)
{
  for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
      i += gridDim.x * blockDim.x)
    out[i] = in[map[i]];
}

static int grid_for(int n, int threads = 256)
{
  int b = (n + threads - 1) / threads;
  return b < 1 ? 1 : (b > 148 * 16 ? 148 * 16 : b);
}

// FP32 -> BF16 bits, round to nearest even (finite inputs)
static uint16_t bf16_round(float f)
{
  uint32_t u;
  std::memcpy(&u, &f, 4);
  u += 0x7FFFu + ((u >> 16) & 1u);
  return (uint16_t)(u >> 16);
}

static float bf16_value(uint16_t h)
{
  const uint32_t u = (uint32_t)h << 16;
  float f;
  std::memcpy(&f, &u, 4);
  return f;
}

void to_full(icarat_ctx *c, const double *in, double *full_out, bool host_src)
{
  const double *src = in;
  if(host_src)
  {
    ICK(cudaMemcpyAsync(c->d_v2, in, sizeof(double) * c->numeq,
                        cudaMemcpyHostToDevice, c->stream));
    src = c->d_v2;
  }
  ICK(cudaMemsetAsync(full_out, 0, sizeof(double) * c->neq, c->stream));
  if(c->numeq > 0)
  {
    note_launch();
    k_scatter_free<<<grid_for(c->numeq), 256, 0, c->stream>>>(c->numeq, c->d_free,
                                                              src, full_out);
  }
  ICK(cudaGetLastError());
}

void from_full(icarat_ctx *c, const double *full_in, double *out, bool host_dst)
{
  double *dst = host_dst ? c->d_v2 : out;
  if(c->numeq > 0)
  {
    note_launch();
    k_gather_free<<<grid_for(c->numeq), 256, 0, c->stream>>>(c->numeq, c->d_free,
                                                             full_in, dst);
  }
  ICK(cudaGetLastError());
  if(host_dst)
  {
    ICK(cudaMemcpyAsync(out, c->d_v2, sizeof(double) * c->numeq,
                        cudaMemcpyDeviceToHost, c->stream));
    ICK(cudaStreamSynchronize(c->stream));
  }
}

int abi_nelx(const icarat_ctx *c) { return c->sel ? c->nelx_sel : c->nelx; }

void elem_in(icarat_ctx *c, const double *src, bool host_src, double *d_box)
{
  if(!c->sel)
  {
    if(src != d_box)
      ICK(cudaMemcpyAsync(d_box, src, sizeof(double) * c->nelx,
                          host_src ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice,
                          c->stream));
    return;
  }
  const double *in = src;
  if(host_src)
  {
    ICK(cudaMemcpyAsync(c->d_sel_buf, src, sizeof(double) * c->nelx_sel,
                        cudaMemcpyHostToDevice, c->stream));
    in = c->d_sel_buf;
  }
  ICK(cudaMemsetAsync(d_box, 0, sizeof(double) * c->nelx, c->stream));
  if(c->nelx_sel > 0)
  {
    note_launch();
    k_sel_scatter<<<grid_for(c->nelx_sel), 256, 0, c->stream>>>(c->nelx_sel, c->d_sel_elem,
                                                                in, d_box);
  }
  ICK(cudaGetLastError());
}

void elem_out(icarat_ctx *c, const double *d_box, double *dst, bool host_dst)
{
  if(!c->sel)
  {
    if(dst != d_box)
      ICK(cudaMemcpyAsync(dst, d_box, sizeof(double) * c->nelx,
                          host_dst ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice,
                          c->stream));
  }
  else
  {
    double *out = host_dst ? c->d_sel_buf : dst;
    if(c->nelx_sel > 0)
    {
      note_launch();
      k_sel_gather<<<grid_for(c->nelx_sel), 256, 0, c->stream>>>(c->nelx_sel,
                                                                 c->d_sel_elem, d_box, out);
    }
    ICK(cudaGetLastError());
    if(host_dst)
      ICK(cudaMemcpyAsync(dst, c->d_sel_buf, sizeof(double) * c->nelx_sel,
                          cudaMemcpyDeviceToHost, c->stream));
  }
  if(host_dst)
    ICK(cudaStreamSynchronize(c->stream));
}

void set_design_device(icarat_ctx *c, const double *d_rho)
{
  if(d_rho != c->d_rho)
    ICK(cudaMemcpyAsync(c->d_rho, d_rho, sizeof(double) * c->nelx,
                        cudaMemcpyDeviceToDevice, c->stream));
  note_launch();
  k_simp<<<grid_for(c->nelx), 256, 0, c->stream>>>(
      c->nelx, c->d_rho, c->mat.young_min, c->mat.young_max, c->mat.penalty,
      c->d_emask, c->d_E, c->d_E32);
  ICK(cudaGetLastError());
  c->design_set = true;
  c->solved = false;
  c->design_version++;
}


// hexa8 faces as SurfaceLoad numbers them (sides 1..6,
// boundary_condition_base.cpp:313-336): local nodes of each face
static const int kFaceNodes[7][4] = {{0, 0, 0, 0}, {0, 1, 2, 3}, {3, 0, 4, 7}, {0, 1, 5, 4},
                                     {1, 2, 6, 5}, {2, 3, 7, 6}, {4, 5, 6, 7}};

// SurfaceLoad::judgeLine for hexa8 (:58-76): the face from the local index k
// of the 4th node inside the load box and the local indices found so far;
// as there, nodes 4,5,6,7 give side 2 (hits[2] - hits[1] == 1 is tested
// first)
static int judge_face(int k, const int *hits)
{
  if(k == 3)
    return 1;
  if(k == 5)
    return 3;
  if(k == 6)
    return 4;
  if(hits[2] - hits[1] == 1)
    return 2;
  if(hits[1] - hits[0] == 1)
    return 5;
  return 6;
}

// equivalent nodal forces of a uniform traction val on a quad4 face X
// (SurfaceLoad::generate :143-187 with snmatrix2d, nmatrix_surface.hpp:60-89):
// fe = sum over the 2 x 2 Gauss points of N^T val |dX/dr1 x dX/dr2|
static void face_load(const double X[4][3], const double *val, double fe[12])
{
  const double g = 1.0 / std::sqrt(3.0);
  const double pts[4][2] = {{-g, -g}, {g, -g}, {-g, g}, {g, g}};
  for(int i = 0; i < 12; i++)
    fe[i] = 0.0;
  for(int ip = 0; ip < 4; ip++)
  {
    const double r0 = pts[ip][0], r1 = pts[ip][1];
    const double N[4] = {0.25 * (1.0 - r0) * (1.0 - r1), 0.25 * (1.0 + r0) * (1.0 - r1),
                         0.25 * (1.0 + r0) * (1.0 + r1), 0.25 * (1.0 - r0) * (1.0 + r1)};
    const double dN[2][4] = {{-0.25 * (1.0 - r1), 0.25 * (1.0 - r1), 0.25 * (1.0 + r1),
                              -0.25 * (1.0 + r1)},
                             {-0.25 * (1.0 - r0), -0.25 * (1.0 + r0), 0.25 * (1.0 + r0),
                              0.25 * (1.0 - r0)}};
    double J[2][3];
    for(int a = 0; a < 2; a++)
      for(int d = 0; d < 3; d++)
      {
        double t = 0.0;
        for(int n = 0; n < 4; n++)
          t += dN[a][n] * X[n][d];
        J[a][d] = t;
      }
    const double cx = J[0][1] * J[1][2] - J[0][2] * J[1][1];
    const double cy = J[0][2] * J[1][0] - J[0][0] * J[1][2];
    const double cz = J[0][0] * J[1][1] - J[0][1] * J[1][0];
    const double jac = std::sqrt(cx * cx + cy * cy + cz * cz) * 1.0;
    for(int n = 0; n < 4; n++)
      for(int d = 0; d < 3; d++)
        fe[3 * n + d] += (N[n] * val[d]) * jac;
  }
}

// global node numbers of element e in the mesher's local order
static void element_nodes(const icarat_ctx *c, long e, long en[8])
{
  const long NX = c->NX, NY = c->NY;
  const long i = e % c->nx, j = (e / c->nx) % c->ny, k = e / ((long)c->nx * c->ny);
  const long b = NX * NY * k + NX * j + i;
  const long o[8] = {0, 1, 1 + NX, NX, NX * NY, 1 + NX * NY, 1 + NX + NX * NY, NX + NX * NY};
  for(int a = 0; a < 8; a++)
    en[a] = b + o[a];
}

// [mesh] selection (MeshIcarat::modifyMesh, src/io/mesh_icarat.hpp:636-755):
// a node is kept when it lies in one of the boxes widened by 1e-7, an element
// when its centroid (the running sum of x / 8 over its local nodes, in that
// order) does; kept nodes and elements keep their box order.  A kept element
// with a removed node is the reference's "error in mesh_icarat" (exit(1)); a
// kept node that no kept element uses would leave a zero stiffness row and is
// refused as well.
static void select_mesh(icarat_ctx *c, int nsel, const double *boxes,
                        std::vector<uint8_t> &keep_node, std::vector<uint8_t> &keep_elem)
{
  const double tol = 1.0e-7;
  const long NX = c->NX, NY = c->NY;
  auto coord = [&](long n, int d) -> double
  {
    long i = n % NX, j = (n / NX) % NY, k = n / (NX * NY);
    if(d == 0)
      return (c->lx / c->nx) * i;
    if(d == 1)
      return (c->ly / c->ny) * j;
    return (c->lz / c->nz) * k;
  };
  keep_node.assign(c->numnp, 0);
  keep_elem.assign(c->nelx, 0);
  for(int b = 0; b < nsel; b++)
  {
    const double *B = boxes + 6 * b;
    const double lo[3] = {B[0] - tol, B[2] - tol, B[4] - tol};
    const double hi[3] = {B[1] + tol, B[3] + tol, B[5] + tol};
    for(long n = 0; n < c->numnp; n++)
    {
      const double x = coord(n, 0), y = coord(n, 1), z = coord(n, 2);
      if(x >= lo[0] && x <= hi[0] && y >= lo[1] && y <= hi[1] && z >= lo[2] && z <= hi[2])
        keep_node[n] = 1;
    }
    for(long e = 0; e < c->nelx; e++)
    {
      long en[8];
      element_nodes(c, e, en);
      double cx = 0.0, cy = 0.0, cz = 0.0;
      for(int a = 0; a < 8; a++)
      {
        cx += coord(en[a], 0) / 8;
        cy += coord(en[a], 1) / 8;
        cz += coord(en[a], 2) / 8;
      }
      if(cx >= lo[0] && cx <= hi[0] && cy >= lo[1] && cy <= hi[1] && cz >= lo[2] &&
         cz <= hi[2])
        keep_elem[e] = 1;
    }
  }
  std::vector<uint8_t> used(c->numnp, 0);
  for(long e = 0; e < c->nelx; e++)
  {
    if(!keep_elem[e])
      continue;
    long en[8];
    element_nodes(c, e, en);
    for(int a = 0; a < 8; a++)
    {
      IREQUIRE(keep_node[en[a]], ICARAT_ERR_ARG,
               "selection keeps element " + std::to_string(e) + " but not its node " +
                   std::to_string(en[a]) + " (error in mesh_icarat)");
      used[en[a]] = 1;
    }
  }
  for(long n = 0; n < c->numnp; n++)
    IREQUIRE(!keep_node[n] || used[n], ICARAT_ERR_ARG,
             "selection keeps node " + std::to_string(n) +
                 " but no element around it (zero stiffness row)");
}

// Mesh + BC on the host, mirroring MeshIcarat/BCIcarat:
//  node coordinates x = (L / div) * index (mesh_icarat.hpp:468-476);
//  Dirichlet boxes widened by 1e-7, flags kept once 1, values overwritten
//  (boundary_condition_icarat.hpp:73-138, boundary_condition_base.hpp:19-33);
//  countDOF numbering (boundary_condition_base.hpp:35-95);
//  point loads on free components of nodes in the widened box
//  (boundary_condition_icarat.hpp:213-264, 380-396).
// With a selection (keep_node / keep_elem non-null) the boundary conditions
// see the kept nodes and elements only, as they see the reference's
// modified mesh; removed nodes get every component fixed and no number.
static void build_mesh_bc(icarat_ctx *c, const icarat_bc *bc,
                          const std::vector<uint8_t> *keep_node = nullptr,
                          const std::vector<uint8_t> *keep_elem = nullptr)
{
  auto kept = [&](long n) { return !keep_node || (*keep_node)[n] != 0; };
  const double tol = 1.0e-7;
  const long NX = c->NX, NY = c->NY;
  auto coord = [&](long n, int d) -> double
  {
    long i = n % NX, j = (n / NX) % NY, k = n / (NX * NY);
    if(d == 0)
      return (c->lx / c->nx) * i;
    if(d == 1)
      return (c->ly / c->ny) * j;
    return (c->lz / c->nz) * k;
  };
  std::vector<uint8_t> has(c->numnp, 0);
  std::vector<int> flag(3 * (size_t)c->numnp, 0);
  std::vector<double> val(3 * (size_t)c->numnp, 0.0);
  for(int d = 0; d < (bc ? bc->n_dirichlet : 0); d++)
  {
    const icarat_dirichlet &D = bc->dirichlet[d];
    for(int q = 0; q < 3; q++)
      IREQUIRE(D.flag[q] == 0 || D.flag[q] == 1, ICARAT_ERR_ARG,
               "dirichlet flags must be 0 or 1");
    // index range of nodes inside the widened box along each axis
    long lo[3], hi[3];
    const int nn[3] = {c->NX, c->NY, c->NZ};
    const double h[3] = {c->lx / c->nx, c->ly / c->ny, c->lz / c->nz};
    for(int a = 0; a < 3; a++)
    {
      lo[a] = nn[a];
      hi[a] = -1;
      for(long i = 0; i < nn[a]; i++)
      {
        double x = h[a] * i;
        if(x >= D.box[a][0] - tol && x <= D.box[a][1] + tol)
        {
          if(i < lo[a])
            lo[a] = i;
          hi[a] = i;
        }
      }
    }
    for(long k = lo[2]; k <= hi[2]; k++)
      for(long j = lo[1]; j <= hi[1]; j++)
        for(long i = lo[0]; i <= hi[0]; i++)
        {
          long n = i + j * NX + k * NX * NY;
          if(!kept(n))
            continue;
          has[n] = 1;
          for(int q = 0; q < 3; q++)
          {
            if(flag[3 * n + q] != 1)
              flag[3 * n + q] = D.flag[q];
            val[3 * n + q] = D.val[q];
          }
        }
  }
  c->dof.assign(3 * (size_t)c->numnp, -1);
  c->fix_h.assign(c->numnp, 0);
  c->uD_h.assign(3 * (size_t)c->numnp, 0.0);
  int counter = 0;
  for(long n = 0; n < c->numnp; n++)
    if(kept(n))
      for(int q = 0; q < 3; q++)
        if(!has[n] || flag[3 * n + q] == 0)
          c->dof[3 * n + q] = counter++;
  c->numeq = counter;
  for(long n = 0; n < c->numnp; n++)
    if(!kept(n))
    {
      // removed node: no equation, no number
      c->fix_h[n] = 7;
      for(int q = 0; q < 3; q++)
        c->dof[3 * n + q] = INT32_MAX;
    }
  for(long n = 0; n < c->numnp; n++)
    if(has[n])
      for(int q = 0; q < 3; q++)
        if(flag[3 * n + q] != 0)
        {
          c->dof[3 * n + q] = counter++;
          c->fix_h[n] |= (uint8_t)(1u << q);
          if(flag[3 * n + q] == 1)
            c->uD_h[3 * n + q] = val[3 * n + q];
          if(c->uD_h[3 * n + q] != 0.0)
            c->has_uD = true;
        }
  // Neumann loads in input order (generateLoadMain,
  // boundary_condition_icarat.hpp:271-410)
  c->fext_h.assign(c->numeq, 0.0);
  for(int l = 0; l < (bc ? bc->n_loads : 0); l++)
  {
    const icarat_load &L = bc->loads[l];
    auto inside = [&](long n) {
      const double x = coord(n, 0), y = coord(n, 1), z = coord(n, 2);
      return L.box[0][0] - tol <= x && x <= L.box[0][1] + tol && L.box[1][0] - tol <= y &&
             y <= L.box[1][1] + tol && L.box[2][0] - tol <= z && z <= L.box[2][1] + tol;
    };
    if(L.box[0][0] == L.box[0][1] && L.box[1][0] == L.box[1][1] && L.box[2][0] == L.box[2][1])
    {
      // point load (:380-396)
      for(long n = 0; n < c->numnp; n++)
        if(kept(n) && inside(n))
          for(int q = 0; q < 3; q++)
          {
            int d = c->dof[3 * n + q];
            if(d < c->numeq)
              c->fext_h[d] += L.val[q];
          }
      continue;
    }
    // distributed load (:336-378): the face of each element found by its
    // nodes inside the box, equivalent nodal forces of the traction L.val
    for(long e = 0; e < c->nelx; e++)
    {
      if(keep_elem && !(*keep_elem)[e])
        continue;
      long en[8];
      element_nodes(c, e, en);
      int hits[8], count = 0;
      for(int k = 0; k < 8; k++)
      {
        if(!inside(en[k]))
          continue;
        hits[count++] = k;
        if(count != 4)
          continue;
        const int *fn = kFaceNodes[judge_face(k, hits)];
        double X[4][3], fe[12];
        for(int i = 0; i < 4; i++)
          for(int d = 0; d < 3; d++)
            X[i][d] = coord(en[fn[i]], d);
        face_load(X, L.val, fe);
        for(int i = 0; i < 4; i++)
          for(int q = 0; q < 3; q++)
          {
            int d = c->dof[3 * en[fn[i]] + q];
            if(d < c->numeq)
              c->fext_h[d] += fe[3 * i + q];
          }
      }
    }
  }
}

} // namespace icarat_b200

using namespace icarat_b200;

int icarat_ctx_create_sel_impl(const icarat_grid *grid, const icarat_material *mat,
                               const icarat_bc *bc, int nsel, const double *boxes,
                               int device, icarat_ctx **out);

int icarat_ctx_create_impl(const icarat_grid *grid, const icarat_material *mat,
                           const icarat_bc *bc, int device, icarat_ctx **out)
{
  return icarat_ctx_create_sel_impl(grid, mat, bc, 0, nullptr, device, out);
}

// nsel > 0: the [mesh] selection boxes (x0, x1, y0, y1, z0, z1 each)
int icarat_ctx_create_sel_impl(const icarat_grid *grid, const icarat_material *mat,
                               const icarat_bc *bc, int nsel, const double *boxes,
                               int device, icarat_ctx **out)
{
  IREQUIRE(grid && mat && out, ICARAT_ERR_ARG, "null argument");
  IREQUIRE(nsel >= 0 && (nsel == 0 || boxes), ICARAT_ERR_ARG, "bad selection");
  IREQUIRE(grid->nx >= 1 && grid->ny >= 1 && grid->nz >= 1, ICARAT_ERR_ARG,
           "division must be >= 1");
  IREQUIRE(grid->lx > 0 && grid->ly > 0 && grid->lz > 0, ICARAT_ERR_ARG,
           "length must be > 0");
  IREQUIRE(mat->young_max - mat->young_min >= 0.0, ICARAT_ERR_ARG,
           "young = [E1, E2] needs E2 >= E1 (elasticity.hpp:15)");
  IREQUIRE(mat->poisson > -1.0 && mat->poisson < 0.5, ICARAT_ERR_ARG,
           "poisson out of range");
  long long numnp = (long long)(grid->nx + 1) * (grid->ny + 1) * (grid->nz + 1);
  IREQUIRE(3 * numnp < (1LL << 31) - 1, ICARAT_ERR_UNSUPPORTED,
           "more than 2^31-1 DOFs");
  icarat_ctx *c = new icarat_ctx();
  try
  {
    c->device = device;
    ICK(cudaSetDevice(device));
    ICK(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    c->nx = grid->nx;
    c->ny = grid->ny;
    c->nz = grid->nz;
    c->lx = grid->lx;
    c->ly = grid->ly;
    c->lz = grid->lz;
    c->hx = grid->lx / grid->nx;
    c->hy = grid->ly / grid->ny;
    c->hz = grid->lz / grid->nz;
    c->NX = c->nx + 1;
    c->NY = c->ny + 1;
    c->NZ = c->nz + 1;
    c->numnp = (int)numnp;
    c->nelx = c->nx * c->ny * c->nz;
    c->neq = 3 * c->numnp;
    c->mat = *mat;
    hexa8_stiffness(c->hx, c->hy, c->hz, mat->poisson, c->ke0.k, &c->vol0);
    hexa8_stress_operator(c->hx, c->hy, c->hz, mat->poisson, c->sb0.s);
    for(int q = 0; q < 576; q++)
      c->ke0f.k[q] = (float)c->ke0.k[q];
    c->ke_diag_max = 0.0;
    for(int a = 0; a < 24; a++)
      c->ke_diag_max = std::fmax(c->ke_diag_max, c->ke0.k[25 * a]);
    c->lam_max_dk = jacobi_bound(c->ke0.k);
    if(nsel > 0)
    {
      std::vector<uint8_t> keep_node, keep_elem;
      select_mesh(c, nsel, boxes, keep_node, keep_elem);
      build_mesh_bc(c, bc, &keep_node, &keep_elem);
      c->sel = true;
      for(long n = 0; n < c->numnp; n++)
        if(keep_node[n])
          c->sel_node_h.push_back((int)n);
      for(long e = 0; e < c->nelx; e++)
        if(keep_elem[e])
          c->sel_elem_h.push_back((int)e);
      c->numnp_sel = (int)c->sel_node_h.size();
      c->nelx_sel = (int)c->sel_elem_h.size();
      IREQUIRE(c->nelx_sel > 0, ICARAT_ERR_ARG, "the selection keeps no element");
      ICK(cudaMalloc(&c->d_emask, c->nelx));
      ICK(cudaMemcpy(c->d_emask, keep_elem.data(), c->nelx, cudaMemcpyHostToDevice));
      ICK(cudaMalloc(&c->d_sel_elem, sizeof(int) * c->nelx_sel));
      ICK(cudaMemcpy(c->d_sel_elem, c->sel_elem_h.data(), sizeof(int) * c->nelx_sel,
                     cudaMemcpyHostToDevice));
      c->d_sel_buf = dalloc(c->nelx_sel);
    }
    else
      build_mesh_bc(c, bc);
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    c->sm_count = sms;
    {
      // Ke0 = hi + lo in BF16 (round to nearest even), zero-padded to 32 x 32
      std::vector<uint16_t> keb(2 * 32 * 32, 0);
      for(int n = 0; n < 24; n++)
        for(int k = 0; k < 24; k++)
        {
          const double v = c->ke0.k[n * 24 + k];
          const uint16_t hi = bf16_round((float)v);
          keb[n * 32 + k] = hi;
          keb[1024 + n * 32 + k] = bf16_round((float)(v - (double)bf16_value(hi)));
        }
      ICK(cudaMalloc(&c->d_keb, sizeof(uint16_t) * keb.size()));
      ICK(cudaMemcpy(c->d_keb, keb.data(), sizeof(uint16_t) * keb.size(),
                     cudaMemcpyHostToDevice));
      ICK(cudaMalloc(&c->d_tc_err, sizeof(int)));
      ICK(cudaMemset(c->d_tc_err, 0, sizeof(int)));
    }
    // streaming CG kernels at full occupancy (8 blocks of 256 threads per
    // SM): with 4 per SM they reached 3-4 TB/s on the B200
    c->red_blocks = sms * 8 > kMaxRedBlocks ? kMaxRedBlocks : sms * 8;
    // icarat_solve_noalloc's buffer: its address is taken here, where the
    // context allocates anyway, so that the solve itself never loads a module
    noalloc_resolve(c);

    // free-DOF map: equation number -> 3 node + component
    std::vector<int> freeidx(c->numeq > 0 ? c->numeq : 1);
    for(long n = 0; n < c->numnp; n++)
      for(int q = 0; q < 3; q++)
        if(c->dof[3 * n + q] < c->numeq)
          freeidx[c->dof[3 * n + q]] = (int)((long)q * c->numnp + n);
    ICK(cudaMalloc(&c->d_free, sizeof(int) * freeidx.size()));
    ICK(cudaMemcpy(c->d_free, freeidx.data(), sizeof(int) * freeidx.size(),
                   cudaMemcpyHostToDevice));
    ICK(cudaMalloc(&c->d_fix, c->numnp));
    ICK(cudaMemcpy(c->d_fix, c->fix_h.data(), c->numnp, cudaMemcpyHostToDevice));
    const size_t nv = (size_t)c->neq;
    c->d_fext = dalloc(nv);
    c->d_rhs = dalloc(nv);
    c->d_u = dalloc(nv);
    c->d_invd = dalloc(nv);
    c->d_r = dalloc(nv);
    c->d_p = dalloc(nv);
    c->d_z = dalloc(nv);
    c->d_Ap = dalloc(nv);
    c->d_v1 = dalloc(nv);
    c->d_v2 = dalloc(nv);
    c->d_rho = dalloc(c->nelx);
    c->d_E = dalloc(c->nelx);
    ICK(cudaMalloc(&c->d_E32, sizeof(float) * (c->nelx > 0 ? c->nelx : 1)));
    c->d_e1 = dalloc(c->nelx);
    c->d_e2 = dalloc(c->nelx);
    c->d_partials = dalloc((size_t)kMaxRedBlocks * 8);
    c->d_scalar = dalloc(64);
    ICK(cudaMalloc(&c->d_counter, sizeof(unsigned int) * 16));
    ICK(cudaMemset(c->d_counter, 0, sizeof(unsigned int) * 16));
    ICK(cudaMalloc(&c->d_cg, sizeof(CgScalars)));
    ICK(cudaMemset(c->d_cg, 0, sizeof(CgScalars)));
    ICK(cudaMallocHost(&c->h_cg, sizeof(CgScalars)));
    ICK(cudaMallocHost(&c->h_scalar, sizeof(double) * 64));
    if(c->has_uD)
    {
      c->d_uD = dalloc(nv);
      std::vector<double> uD(nv);
      for(long n = 0; n < c->numnp; n++)
        for(int q = 0; q < 3; q++)
          uD[(long)q * c->numnp + n] = c->uD_h[3 * n + q];
      ICK(cudaMemcpy(c->d_uD, uD.data(), sizeof(double) * nv, cudaMemcpyHostToDevice));
    }
    ICK(cudaMemset(c->d_u, 0, sizeof(double) * nv));
    // fext in node layout
    std::vector<double> ff(nv, 0.0);
    for(long n = 0; n < c->numnp; n++)
      for(int q = 0; q < 3; q++)
        if(c->dof[3 * n + q] < c->numeq)
          ff[(long)q * c->numnp + n] = c->fext_h[c->dof[3 * n + q]];
    ICK(cudaMemcpy(c->d_fext, ff.data(), sizeof(double) * nv,
                   cudaMemcpyHostToDevice));
  }
  catch(...)
  {
    icarat_ctx_destroy(c);
    throw;
  }
  *out = c;
  return ICARAT_OK;
}

int icarat_ctx_destroy_impl(icarat_ctx *c)
{
  if(!c)
    return ICARAT_OK;
  cudaSetDevice(c->device);
  if(c->stream)
    cudaStreamSynchronize(c->stream);
  mg_free(c);
  mixed_free(c);
  filter_free(c);
  helm_free(c);
  if(c->loop.mma)
    icarat_mma_destroy(c->loop.mma);
  for(double *p : {c->loop.x, c->loop.xfil, c->loop.xthr, c->loop.thrd,
                   c->loop.dfds, c->loop.dgds, c->loop.tmp, c->loop.tmp2, c->loop.xmin,
                   c->loop.xmax, c->loop.d_cases, c->loop.d_cases_u, c->loop.d_volw})
    dfree(p);
  dfree(c->loop.d_fixed);
  dfree(c->loop.d_sel);
  dfree(c->d_emask);
  dfree(c->d_sel_elem);
  dfree(c->d_sel_buf);
  dfree(c->d_free);
  dfree(c->d_fix);
  dfree(c->d_uD);
  for(double *p : {c->d_fext, c->d_rhs, c->d_u, c->d_invd, c->d_r, c->d_p,
                   c->d_z, c->d_Ap, c->d_v1, c->d_v2, c->d_rho, c->d_E,
                   c->d_e1, c->d_e2, c->d_partials, c->d_scalar, c->d_stage})
    dfree(p);
  dfree(c->d_counter);
  dfree(c->d_cg);
  dfree(c->d_keb);
  dfree(c->d_E32);
  dfree(c->d_tc_err);
  if(c->h_cg)
    cudaFreeHost(c->h_cg);
  if(c->h_scalar)
    cudaFreeHost(c->h_scalar);
  if(c->stream)
    cudaStreamDestroy(c->stream);
  delete c;
  return ICARAT_OK;
}
