// Legacy VTK output of the voxel box (src/io/export_vtk.hpp, as the sample
// drivers' output(): opt_macro_mma_nondesign.cpp:220-242).
//
// ASCII files are written exactly as the reference writes them: the header
// of makeHeaderVTK (:47-53), POINTS / CELLS / CELL_TYPES of setPointVTK,
// setElementVTK and setElementTypeVTK (:67-112), then the point vector
// "displacement" and the cell scalars "density" and "mises"
// (addPointVectorVTK :134-151, addElementScalarVTK :153-170), every number
// through an ostream with its default formatting, tab separated, as there.
// Node positions are (lx / nx) i, (ly / ny) j, (lz / nz) k and cells list the
// hexa8 nodes in the mesher's order (VTK cell type 12).  With binary != 0 the
// same sections are written as legacy BINARY (big-endian float32 / int32),
// which for a 2M-element box is a 100 MB file written at disk speed instead
// of formatted text.
#include <cstdint>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

#include "internal.cuh"

namespace icarat_b200
{
namespace
{

struct Box
{
  int nx, ny, nz;
  double lx, ly, lz;
  long NX, NY, NZ, numnp, nelx;
};

void put_be32(std::ofstream &f, uint32_t v)
{
  const char b[4] = {(char)(v >> 24), (char)(v >> 16), (char)(v >> 8), (char)v};
  f.write(b, 4);
}

void put_f32(std::ofstream &f, double v)
{
  const float x = (float)v;
  uint32_t u;
  std::memcpy(&u, &x, 4);
  put_be32(f, u);
}

void node_of_cell(const Box &b, long e, long c[8])
{
  const long i = e % b.nx, j = (e / b.nx) % b.ny, k = e / ((long)b.nx * b.ny);
  const long n = b.NX * b.NY * k + b.NX * j + i;
  c[0] = n;
  c[1] = n + 1;
  c[2] = n + 1 + b.NX;
  c[3] = n + b.NX;
  c[4] = n + b.NX * b.NY;
  c[5] = n + 1 + b.NX * b.NY;
  c[6] = n + 1 + b.NX + b.NX * b.NY;
  c[7] = n + b.NX + b.NX * b.NY;
}

} // namespace

void write_vtk(const char *path, bool binary, int nx, int ny, int nz, double lx, double ly,
               double lz, const double *node_val, const double *density, const double *mises)
{
  IREQUIRE(path && nx >= 1 && ny >= 1 && nz >= 1, ICARAT_ERR_ARG, "bad VTK arguments");
  Box b{nx, ny, nz, lx, ly, lz, nx + 1, ny + 1, nz + 1, 0, 0};
  b.numnp = b.NX * b.NY * b.NZ;
  b.nelx = (long)nx * ny * nz;
  std::ofstream f(path, std::ios::out | std::ios::trunc | std::ios::binary);
  IREQUIRE(f.good(), ICARAT_ERR_ARG, std::string("cannot open ") + path);
  const double hx = lx / nx, hy = ly / ny, hz = lz / nz;
  f << "# vtk DataFile Version 4.1\n";
  f << "vtk output\n";
  f << (binary ? "BINARY\n" : "ASCII\n");
  f << "DATASET UNSTRUCTURED_GRID\n";
  // points
  f << "\nPOINTS\t" << b.numnp << "\tfloat\n";
  for(long k = 0; k < b.NZ; k++)
    for(long j = 0; j < b.NY; j++)
      for(long i = 0; i < b.NX; i++)
      {
        const double x[3] = {hx * i, hy * j, hz * k};
        if(binary)
          for(int d = 0; d < 3; d++)
            put_f32(f, x[d]);
        else
        {
          for(int d = 0; d < 3; d++)
            f << x[d] << "\t";
          f << '\n'; // the reference's std::endl without its flush
        }
      }
  if(binary)
    f << "\n";
  // cells and their types
  f << "\nCELLS " << b.nelx << "\t" << 9 * b.nelx << "\n";
  for(long e = 0; e < b.nelx; e++)
  {
    long c[8];
    node_of_cell(b, e, c);
    if(binary)
    {
      put_be32(f, 8u);
      for(int a = 0; a < 8; a++)
        put_be32(f, (uint32_t)c[a]);
    }
    else
    {
      f << 8 << "\t";
      for(int a = 0; a < 8; a++)
        f << c[a] << "\t";
      f << '\n'; // the reference's std::endl without its flush
    }
  }
  if(binary)
    f << "\n";
  f << "\nCELL_TYPES\t" << b.nelx << "\n";
  for(long e = 0; e < b.nelx; e++)
  {
    if(binary)
      put_be32(f, 12u);
    else
      f << 12 << "\n";
  }
  if(binary)
    f << "\n";
  // displacement at the nodes
  if(node_val)
  {
    f << "\nPOINT_DATA\t" << b.numnp << "\n";
    f << "VECTORS displacement float\n";
    for(long n = 0; n < b.numnp; n++)
    {
      if(binary)
        for(int d = 0; d < 3; d++)
          put_f32(f, node_val[3 * n + d]);
      else
      {
        for(int d = 0; d < 3; d++)
          f << node_val[3 * n + d] << "\t";
        f << '\n'; // the reference's std::endl without its flush
      }
    }
    if(binary)
      f << "\n";
  }
  // element scalars
  bool header = true;
  const char *names[2] = {"density", "mises"};
  const double *fields[2] = {density, mises};
  for(int q = 0; q < 2; q++)
  {
    if(!fields[q])
      continue;
    if(header)
      f << "\nCELL_DATA\t" << b.nelx << "\n";
    header = false;
    f << "SCALARS " << names[q] << " float\n";
    f << "LOOKUP_TABLE default\n";
    for(long e = 0; e < b.nelx; e++)
    {
      if(binary)
        put_f32(f, fields[q][e]);
      else
        f << fields[q][e] << '\n';
    }
    if(binary)
      f << "\n";
  }
  f.close();
  IREQUIRE(!f.fail(), ICARAT_ERR_ARG, std::string("writing ") + path + " failed");
}

} // namespace icarat_b200
