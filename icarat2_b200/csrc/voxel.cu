// STL surface -> voxel design domain (the role of scripts/stl_to_vtk_voxel.py,
// which marks the cells of a mesh_size^3 grid over the surface's bounding box
// whose centres vtkSelectEnclosedPoints finds inside the closed surface).
//
// Here the inside test is ray parity along +z, per column of voxel centres:
// every crossing of the vertical line through a column centre (x, y) with a
// triangle is recorded, the column's crossings are sorted, and a voxel centre
// is inside when an odd number of crossings lie below it.  A CTA per triangle
// walks the columns under the triangle's xy bounding box (so the work is
// proportional to the projected area, not columns x triangles); a thread per
// column then sorts its crossings and fills its voxels with coalesced stores.
// Points on a shared edge or vertex of the xy projection belong to exactly
// one triangle of a consistently oriented sheet: edges are half-open by a
// top-left rule on counter-clockwise projected triangles, and an edge's
// function is evaluated from its smaller endpoint so that the two triangles
// sharing it see exactly opposite values.  Triangles whose
// projection has zero area (parallel to z) never cross a vertical line
// through their interior and are skipped.
#include <cmath>
#include <vector>

#include "internal.cuh"

namespace icarat_b200
{
namespace
{

constexpr int kVoxCap = 256; // crossings kept per column

struct VoxGrid
{
  int nx, ny, nz;
  double ox, oy, oz; // lower corner
  double px, py, pz; // pitch
};

// edge function of the projected edge a -> b at p
__host__ __device__ inline double edge_fn(double ax, double ay, double bx, double by, double px,
                                          double py)
{
  return (bx - ax) * (py - ay) - (by - ay) * (px - ax);
}

// the same value, negated, whichever way round a shared edge is passed:
// evaluated from its lexicographically smaller endpoint
__host__ __device__ inline double edge_canon(double ax, double ay, double bx, double by, double px,
                                             double py)
{
  const bool swap = (bx < ax) || (bx == ax && by < ay);
  return swap ? -edge_fn(bx, by, ax, ay, px, py) : edge_fn(ax, ay, bx, by, px, py);
}

// whether a zero edge value counts as inside (top-left rule for
// counter-clockwise triangles)
__host__ __device__ inline bool top_left(double ax, double ay, double bx, double by)
{
  // for a counter-clockwise triangle: a top edge runs in -x exactly
  // horizontally, a left edge runs downwards
  return (ay == by && bx < ax) || (by < ay);
}

__global__ void k_vox_cross(const double *__restrict__ tri, int ntri, VoxGrid g,
                            double *__restrict__ zs, int *__restrict__ cnt, int *overflow)
{
  for(int t = blockIdx.x; t < ntri; t += gridDim.x)
  {
    const double *v = tri + 9L * t;
    double ax = v[0], ay = v[1], az = v[2];
    double bx = v[3], by = v[4], bz = v[5];
    double cx = v[6], cy = v[7], cz = v[8];
    double area = edge_fn(ax, ay, bx, by, cx, cy);
    if(area == 0.0)
      continue;
    if(area < 0.0)
    {
      // counter-clockwise in xy
      double tx = bx, ty = by, tz = bz;
      bx = cx;
      by = cy;
      bz = cz;
      cx = tx;
      cy = ty;
      cz = tz;
      area = -area;
    }
    const double xmin = fmin(ax, fmin(bx, cx)), xmax = fmax(ax, fmax(bx, cx));
    const double ymin = fmin(ay, fmin(by, cy)), ymax = fmax(ay, fmax(by, cy));
    // columns whose centre ox + (i + 1/2) px lies in [xmin, xmax]
    const int i0 = max(0, (int)ceil((xmin - g.ox) / g.px - 0.5));
    const int i1 = min(g.nx - 1, (int)floor((xmax - g.ox) / g.px - 0.5));
    const int j0 = max(0, (int)ceil((ymin - g.oy) / g.py - 0.5));
    const int j1 = min(g.ny - 1, (int)floor((ymax - g.oy) / g.py - 0.5));
    if(i1 < i0 || j1 < j0)
      continue;
    const bool tl0 = top_left(bx, by, cx, cy), tl1 = top_left(cx, cy, ax, ay),
               tl2 = top_left(ax, ay, bx, by);
    const int wi = i1 - i0 + 1;
    const long ncols = (long)wi * (j1 - j0 + 1);
    for(long q = threadIdx.x; q < ncols; q += blockDim.x)
    {
      const int i = i0 + (int)(q % wi), j = j0 + (int)(q / wi);
      const double px = g.ox + (i + 0.5) * g.px, py = g.oy + (j + 0.5) * g.py;
      const double w0 = edge_canon(bx, by, cx, cy, px, py);
      const double w1 = edge_canon(cx, cy, ax, ay, px, py);
      const double w2 = edge_canon(ax, ay, bx, by, px, py);
      const bool in = (w0 > 0.0 || (w0 == 0.0 && tl0)) && (w1 > 0.0 || (w1 == 0.0 && tl1)) &&
                      (w2 > 0.0 || (w2 == 0.0 && tl2));
      if(!in)
        continue;
      const double z = (w0 * az + w1 * bz + w2 * cz) / area;
      const long col = i + (long)j * g.nx;
      const int pos = atomicAdd(cnt + col, 1);
      if(pos < kVoxCap)
        zs[col * kVoxCap + pos] = z;
      else
        atomicExch(overflow, 1);
    }
  }
}

__global__ void k_vox_fill(VoxGrid g, double *__restrict__ zs, const int *__restrict__ cnt,
                           uint8_t *__restrict__ mask)
{
  const long ncols = (long)g.nx * g.ny;
  for(long col = blockIdx.x * (long)blockDim.x + threadIdx.x; col < ncols;
      col += (long)gridDim.x * blockDim.x)
  {
    double *z = zs + col * kVoxCap;
    const int n = min(cnt[col], kVoxCap);
    // insertion sort of the column's crossings (tens at most in practice)
    for(int a = 1; a < n; a++)
    {
      const double v = z[a];
      int b = a - 1;
      while(b >= 0 && z[b] > v)
      {
        z[b + 1] = z[b];
        b--;
      }
      z[b + 1] = v;
    }
    int below = 0;
    for(int k = 0; k < g.nz; k++)
    {
      const double zc = g.oz + (k + 0.5) * g.pz;
      while(below < n && z[below] < zc)
        below++;
      mask[col + (long)k * ncols] = (uint8_t)(below & 1);
    }
  }
}

} // namespace

// inside (1) / outside (0) of the closed triangle surface tri (ntri x 9:
// three xyz vertices) for the centres of an nx x ny x nz voxel grid with lower
// corner origin and the given pitch; mask is a host array of nx ny nz bytes,
// x fastest
void voxelize(int device, const double *tri, int ntri, int nx, int ny, int nz,
              const double *origin, const double *pitch, uint8_t *mask)
{
  IREQUIRE(tri && ntri >= 1 && nx >= 1 && ny >= 1 && nz >= 1 && origin && pitch && mask,
           ICARAT_ERR_ARG, "bad voxelize arguments");
  IREQUIRE(pitch[0] > 0 && pitch[1] > 0 && pitch[2] > 0, ICARAT_ERR_ARG,
           "voxel pitch must be positive");
  for(long q = 0; q < 9L * ntri; q++)
    IREQUIRE(std::isfinite(tri[q]), ICARAT_ERR_ARG, "non-finite triangle coordinate");
  ICK(cudaSetDevice(device));
  const long ncols = (long)nx * ny, nvox = ncols * nz;
  VoxGrid g{nx, ny, nz, origin[0], origin[1], origin[2], pitch[0], pitch[1], pitch[2]};
  double *d_tri = nullptr, *d_zs = nullptr;
  int *d_cnt = nullptr, *d_over = nullptr;
  uint8_t *d_mask = nullptr;
  cudaStream_t st = nullptr;
  auto release = [&]() {
    cudaFree(d_tri);
    cudaFree(d_zs);
    cudaFree(d_cnt);
    cudaFree(d_over);
    cudaFree(d_mask);
    if(st)
      cudaStreamDestroy(st);
  };
  try
  {
    ICK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    ICK(cudaMalloc(&d_tri, sizeof(double) * 9 * (size_t)ntri));
    ICK(cudaMalloc(&d_zs, sizeof(double) * kVoxCap * (size_t)ncols));
    ICK(cudaMalloc(&d_cnt, sizeof(int) * (size_t)ncols));
    ICK(cudaMalloc(&d_over, sizeof(int)));
    ICK(cudaMalloc(&d_mask, (size_t)nvox));
    ICK(cudaMemcpyAsync(d_tri, tri, sizeof(double) * 9 * (size_t)ntri, cudaMemcpyHostToDevice,
                        st));
    ICK(cudaMemsetAsync(d_cnt, 0, sizeof(int) * (size_t)ncols, st));
    ICK(cudaMemsetAsync(d_over, 0, sizeof(int), st));
    int sms = 148;
    ICK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    note_launch(2);
    k_vox_cross<<<ntri < 64 * sms ? ntri : 64 * sms, 128, 0, st>>>(d_tri, ntri, g, d_zs, d_cnt,
                                                                   d_over);
    ICK(cudaGetLastError());
    const long fb = (ncols + 127) / 128;
    k_vox_fill<<<(int)(fb < 16 * sms ? fb : 16 * sms), 128, 0, st>>>(g, d_zs, d_cnt, d_mask);
    ICK(cudaGetLastError());
    int over = 0;
    ICK(cudaMemcpyAsync(&over, d_over, sizeof(int), cudaMemcpyDeviceToHost, st));
    ICK(cudaMemcpyAsync(mask, d_mask, (size_t)nvox, cudaMemcpyDeviceToHost, st));
    ICK(cudaStreamSynchronize(st));
    IREQUIRE(!over, ICARAT_ERR_UNSUPPORTED,
             "more than 256 surface crossings on one voxel column");
  }
  catch(...)
  {
    release();
    throw;
  }
  release();
}

} // namespace icarat_b200
