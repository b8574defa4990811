/*
 * icarat_oracle.c -- CPU restatement of ICARAT2's linear-static SIMP
 * topology-optimisation loop (hexa8 voxel mesh, SIMP, Jacobi-PCG, radius
 * density filter, OC and MMA updates).
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA library in
 * icarat2_b200/.  Only tests/, __graft_entry__.smoke() and the CPU-baseline
 * leg of bench.py load it; the product path never calls it.
 *
 * Every function cites the reference file:line it restates (paths relative to
 * the ICARAT2 source tree).  Pinning of this restatement:
 *   - distance filter forward/transposed/sensitivity filter against the
 *     known answers of sample/test/test-optimization/test_filter.cpp:63-124;
 *   - hexa8 unit-cube volume of sample/test/test-basis/test_bmatrix.cpp:123-146;
 *   - MMA against the reference's own MMASolver.cpp compiled from source
 *     (oracle/Makefile -> oracle/_ref) and its toy test
 *     (test_opt_solver.cpp:17-73); OC against the reference OCSolver.hpp;
 *   - the 24x24 element matrix against an independent closed form and the
 *     assembled K / solution against scipy.sparse (tests/test_oracle.py).
 * The structural K.u solve itself has no golden vector in the reference
 * (Eigen is not available here), so that part is pinned by the closed forms
 * above, not by reference outputs.
 *
 * Deliberate differences from the reference, none of which changes a result
 * by more than rounding:
 *   - Ke_e is E(rho_e) * Ke0 with Ke0 integrated once on the first element,
 *     instead of re-integrating B^T D(E) B per element and per assembly;
 *   - K is assembled straight into CSR (duplicates summed in element-colour
 *     order) instead of triplets + setFromTriplets, and only once per solve
 *     (the reference assembles a second time for reaction forces);
 *   - neighbour lists of the filter can be built by grid bucketing; the lists
 *     and their order are identical to the O(N^2) preNeighbour.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define OR_OK 0
#define OR_ERR_ARG -1
#define OR_ERR_STATE -5
#define OR_ERR_FILTER -6
#define OR_ERR_UNSUPPORTED -7

static double or_now(void)
{
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

int or_num_threads(void)
{
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

void or_set_threads(int n)
{
#ifdef _OPENMP
  if(n > 0)
    omp_set_num_threads(n);
#else
  (void)n;
#endif
}

/* ------------------------------------------------------------------------ */
/* 1. Structured hexa8 box mesh: MeshIcarat::setParameter (hexa8 counts,     */
/*    src/io/mesh_icarat.hpp:106-111) and MeshIcarat::meshBox hexa8 branch    */
/*    (src/io/mesh_icarat.hpp:459-512).  Node id = i + j(nx+1) +              */
/*    k(nx+1)(ny+1); element id = i + j nx + k nx ny; local node order        */
/*    0:(0,0,0) 1:(1,0,0) 2:(1,1,0) 3:(0,1,0), 4..7 the same at z+1.          */
/* ------------------------------------------------------------------------ */
void or_mesh_box(int nx, int ny, int nz, double lx, double ly, double lz,
                 double *xyz, int *conn)
{
  const long NX = nx + 1, NY = ny + 1, NZ = nz + 1;
  for(long k = 0; k < NZ; k++)
    for(long j = 0; j < NY; j++)
      for(long i = 0; i < NX; i++)
      {
        long n = i + j * NX + k * NX * NY;
        xyz[3 * n + 0] = (lx / nx) * i;
        xyz[3 * n + 1] = (ly / ny) * j;
        xyz[3 * n + 2] = (lz / nz) * k;
      }
  for(long k = 0; k < nz; k++)
    for(long j = 0; j < ny; j++)
      for(long i = 0; i < nx; i++)
      {
        long e = i + j * nx + k * (long)nx * ny;
        long b = NX * NY * k + NX * j + i;
        int *c = conn + 8 * e;
        c[0] = (int)b;
        c[1] = (int)(b + 1);
        c[2] = (int)(b + 1 + NX);
        c[3] = (int)(b + NX);
        c[4] = (int)(b + NX * NY);
        c[5] = (int)(b + 1 + NX * NY);
        c[6] = (int)(b + 1 + NX + NX * NY);
        c[7] = (int)(b + NX + NX * NY);
      }
}

/* ------------------------------------------------------------------------ */
/* 2. Dirichlet boxes and DOF numbering.                                    */
/*    BCIcarat::input_dirich (src/io/boundary_condition_icarat.hpp:73-138):  */
/*    every node inside [min-1e-7, max+1e-7]^3 of a box gets the box's        */
/*    flags/values through setDirichValue (boundary_condition_base.hpp:19-33: */
/*    a flag already 1 stays 1, values are overwritten by the last box).      */
/*    countDOF (boundary_condition_base.hpp:35-95): free components numbered  */
/*    node-major 0..numeq-1, constrained ones numeq..neq-1 afterwards.        */
/* ------------------------------------------------------------------------ */
int or_count_dof(int numnp, const double *xyz, int ndir, const int *dflag,
                 const double *dval, const double *dbox, int *dof,
                 int *has_dirich, int *node_flag, double *node_dval)
{
  const double tol = 1.0e-7;
  for(int n = 0; n < numnp; n++)
  {
    has_dirich[n] = 0;
    for(int c = 0; c < 3; c++)
    {
      node_flag[3 * n + c] = 0;
      node_dval[3 * n + c] = 0.0;
    }
  }
  for(int d = 0; d < ndir; d++)
  {
    const double *b = dbox + 6 * d;
    double xmn = b[0] - tol, xmx = b[1] + tol;
    double ymn = b[2] - tol, ymx = b[3] + tol;
    double zmn = b[4] - tol, zmx = b[5] + tol;
    for(int n = 0; n < numnp; n++)
    {
      const double *x = xyz + 3 * n;
      if(x[0] >= xmn && x[0] <= xmx && x[1] >= ymn && x[1] <= ymx &&
         x[2] >= zmn && x[2] <= zmx)
      {
        has_dirich[n] = 1;
        for(int c = 0; c < 3; c++)
        {
          if(node_flag[3 * n + c] != 1)
            node_flag[3 * n + c] = dflag[3 * d + c];
          node_dval[3 * n + c] = dval[3 * d + c];
        }
      }
    }
  }
  int counter = 0;
  for(int n = 0; n < numnp; n++)
    for(int c = 0; c < 3; c++)
    {
      dof[3 * n + c] = -1;
      if(!has_dirich[n] || node_flag[3 * n + c] == 0)
        dof[3 * n + c] = counter++;
    }
  int numeq = counter;
  for(int n = 0; n < numnp; n++)
    if(has_dirich[n])
      for(int c = 0; c < 3; c++)
        if(node_flag[3 * n + c] != 0)
          dof[3 * n + c] = counter++;
  return numeq;
}

/* ------------------------------------------------------------------------ */
/* 3. Neumann loads: BCIcarat::input_neumann (boundary_condition_icarat.hpp: */
/*    213-264) marks a box whose three ranges are all degenerate as a point   */
/*    load, anything else as distributed; both are widened by 1e-7.          */
/*    generateLoadMain (:271-410), loads in input order:                     */
/*    point (:380-396): val[c] to fext_org[dof] of every free component of   */
/*    every node inside the box;                                            */
/*    distributed (:336-378): per element, nodes tested in local order; when */
/*    the 4th one inside is found at local index k, SurfaceLoad::judgeLine   */
/*    (boundary_condition_base.cpp:58-76) picks the face from k and the hit  */
/*    list, resizeSurfaceParameter (:313-336) its 4 nodes, and generate       */
/*    (:143-187) adds fe = sum_ip N^T val |dX/dr1 x dX/dr2| over the 2 x 2    */
/*    Gauss points of the quad4 face (snmatrix2d, nmatrix_surface.hpp:60-89; */
/*    Gauss4Square gauss_integration.cpp:72-88; ShapeFunction4Square        */
/*    shape_function.cpp:97-119) to the face nodes' free components.  As in */
/*    the reference, hits at local nodes 4,5,6,7 (the z-max face) select     */
/*    face 2 (nodes 3,0,4,7): judgeLine tests hitpoints[2] - hitpoints[1]    */
/*    == 1 first.                                                            */
/* ------------------------------------------------------------------------ */
static const int or_face_nodes[7][4] = {{0, 0, 0, 0}, {0, 1, 2, 3}, {3, 0, 4, 7}, {0, 1, 5, 4},
                                        {1, 2, 6, 5}, {2, 3, 7, 6}, {4, 5, 6, 7}};

static int or_judge_face(int counter, const int *hits)
{
  if(counter == 3)
    return 1;
  if(counter == 5)
    return 3;
  if(counter == 6)
    return 4;
  if(hits[2] - hits[1] == 1)
    return 2;
  if(hits[1] - hits[0] == 1)
    return 5;
  return 6;
}

static void or_surface_fe(const double X[4][3], const double *val, double fe[12])
{
  const double g = 1.0 / sqrt(3.0);
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
    const double jac = sqrt(cx * cx + cy * cy + cz * cz) * 1.0;
    for(int n = 0; n < 4; n++)
      for(int d = 0; d < 3; d++)
        fe[3 * n + d] += (N[n] * val[d]) * jac;
  }
}

int or_point_loads(int numnp, const double *xyz, const int *dof, int numeq, int nelx,
                   const int *conn, int nload, const double *lval, const double *lbox,
                   double *fext)
{
  const double tol = 1.0e-7;
  (void)numnp;
  for(int i = 0; i < numeq; i++)
    fext[i] = 0.0;
  for(int l = 0; l < nload; l++)
  {
    const double *b = lbox + 6 * l;
    const double *v = lval + 3 * l;
#define OR_IN_BOX(x)                                                                         \
  (b[0] - tol <= (x)[0] && (x)[0] <= b[1] + tol && b[2] - tol <= (x)[1] &&                   \
   (x)[1] <= b[3] + tol && b[4] - tol <= (x)[2] && (x)[2] <= b[5] + tol)
    if(b[0] == b[1] && b[2] == b[3] && b[4] == b[5])
    {
      for(int n = 0; n < numnp; n++)
        if(OR_IN_BOX(xyz + 3 * n))
          for(int c = 0; c < 3; c++)
          {
            int d = dof[3 * n + c];
            if(d < numeq)
              fext[d] += v[c];
          }
      continue;
    }
    for(long e = 0; e < nelx; e++)
    {
      const int *ce = conn + 8 * e;
      int hits[8], count = 0;
      for(int k = 0; k < 8; k++)
      {
        if(!OR_IN_BOX(xyz + 3 * (long)ce[k]))
          continue;
        hits[count++] = k;
        if(count == 4)
        {
          const int *fn = or_face_nodes[or_judge_face(k, hits)];
          double X[4][3], fe[12];
          for(int i = 0; i < 4; i++)
            for(int d = 0; d < 3; d++)
              X[i][d] = xyz[3 * (long)ce[fn[i]] + d];
          or_surface_fe(X, v, fe);
          for(int i = 0; i < 4; i++)
            for(int c = 0; c < 3; c++)
            {
              int d = dof[3 * (long)ce[fn[i]] + c];
              if(d < numeq)
                fext[d] += fe[3 * i + c];
            }
        }
      }
    }
#undef OR_IN_BOX
  }
  return OR_OK;
}

/* ------------------------------------------------------------------------ */
/* 4. hexa8 element stiffness.                                               */
/*    Gauss8Cubic (src/basis/gauss_integration.cpp:268-289): points          */
/*    (+-1/sqrt3)^3 in the order below, weights 1.                           */
/*    ShapeFunction8Cubic::dNdr (src/basis/shape_function.cpp:422-447).      */
/*    bmatrix3d (src/basis/bmatrix.hpp:91-162): dXdr = dNdr X,               */
/*    dNdX = dXdr^-1 dNdr, Voigt rows xx,yy,zz,xy,yz,zx, jac = det * w.       */
/*    Elastic::De 3D (src/problem/elasticity.cpp:72-93).                     */
/*    LinearElastic::makeKeFint (src/problem/elasticity.cpp:211-255):        */
/*    Ke = sum_gp B^T D B jac, volume = sum_gp jac.                          */
/* ------------------------------------------------------------------------ */
static const int or_gauss_sign[8][3] = {{-1, -1, -1}, {1, -1, -1}, {1, 1, -1},
                                        {-1, 1, -1},  {-1, -1, 1}, {1, -1, 1},
                                        {1, 1, 1},    {-1, 1, 1}};

static void or_dNdr(const double r[3], double d[3][8])
{
  const double r0 = r[0], r1 = r[1], r2 = r[2];
  d[0][0] = -0.125 * (1.0 - r1) * (1.0 - r2);
  d[0][1] = 0.125 * (1.0 - r1) * (1.0 - r2);
  d[0][2] = 0.125 * (1.0 + r1) * (1.0 - r2);
  d[0][3] = -0.125 * (1.0 + r1) * (1.0 - r2);
  d[0][4] = -0.125 * (1.0 - r1) * (1.0 + r2);
  d[0][5] = 0.125 * (1.0 - r1) * (1.0 + r2);
  d[0][6] = 0.125 * (1.0 + r1) * (1.0 + r2);
  d[0][7] = -0.125 * (1.0 + r1) * (1.0 + r2);
  d[1][0] = -0.125 * (1.0 - r2) * (1.0 - r0);
  d[1][1] = -0.125 * (1.0 - r2) * (1.0 + r0);
  d[1][2] = 0.125 * (1.0 - r2) * (1.0 + r0);
  d[1][3] = 0.125 * (1.0 - r2) * (1.0 - r0);
  d[1][4] = -0.125 * (1.0 + r2) * (1.0 - r0);
  d[1][5] = -0.125 * (1.0 + r2) * (1.0 + r0);
  d[1][6] = 0.125 * (1.0 + r2) * (1.0 + r0);
  d[1][7] = 0.125 * (1.0 + r2) * (1.0 - r0);
  d[2][0] = -0.125 * (1.0 - r0) * (1.0 - r1);
  d[2][1] = -0.125 * (1.0 + r0) * (1.0 - r1);
  d[2][2] = -0.125 * (1.0 + r0) * (1.0 + r1);
  d[2][3] = -0.125 * (1.0 - r0) * (1.0 + r1);
  d[2][4] = 0.125 * (1.0 - r0) * (1.0 - r1);
  d[2][5] = 0.125 * (1.0 + r0) * (1.0 - r1);
  d[2][6] = 0.125 * (1.0 + r0) * (1.0 + r1);
  d[2][7] = 0.125 * (1.0 - r0) * (1.0 + r1);
}

void or_elastic_D(double E, double nu, double D[36])
{
  double lam = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu));
  double mu = E / (2 * (1.0 + nu));
  for(int i = 0; i < 36; i++)
    D[i] = 0.0;
  for(int i = 0; i < 3; i++)
    for(int j = 0; j < 3; j++)
      D[6 * i + j] = (i == j) ? lam + 2 * mu : lam;
  D[6 * 3 + 3] = mu;
  D[6 * 4 + 4] = mu;
  D[6 * 5 + 5] = mu;
}

/* X: 8x3 node coordinates in local order.  Ke: 24x24 row-major. */
void or_hexa8_ke(const double *X, double E, double nu, double *Ke,
                 double *volume)
{
  const double g = 1.0 / sqrt(3.0);
  double D[36];
  or_elastic_D(E, nu, D);
  for(int i = 0; i < 576; i++)
    Ke[i] = 0.0;
  double vol = 0.0;
  for(int ip = 0; ip < 8; ip++)
  {
    double r[3] = {or_gauss_sign[ip][0] * g, or_gauss_sign[ip][1] * g,
                   or_gauss_sign[ip][2] * g};
    double dN[3][8];
    or_dNdr(r, dN);
    double J[3][3];
    for(int a = 0; a < 3; a++)
      for(int b = 0; b < 3; b++)
      {
        double s = 0.0;
        for(int n = 0; n < 8; n++)
          s += dN[a][n] * X[3 * n + b];
        J[a][b] = s;
      }
    double det = J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) -
                 J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +
                 J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
    double inv[3][3];
    inv[0][0] = (J[1][1] * J[2][2] - J[1][2] * J[2][1]) / det;
    inv[0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) / det;
    inv[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) / det;
    inv[1][0] = (J[1][2] * J[2][0] - J[1][0] * J[2][2]) / det;
    inv[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) / det;
    inv[1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) / det;
    inv[2][0] = (J[1][0] * J[2][1] - J[1][1] * J[2][0]) / det;
    inv[2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) / det;
    inv[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) / det;
    double dX[3][8];
    for(int a = 0; a < 3; a++)
      for(int n = 0; n < 8; n++)
      {
        double s = 0.0;
        for(int b = 0; b < 3; b++)
          s += inv[a][b] * dN[b][n];
        dX[a][n] = s;
      }
    double B[6][24];
    memset(B, 0, sizeof(B));
    for(int n = 0; n < 8; n++)
    {
      B[0][3 * n] = dX[0][n];
      B[1][3 * n + 1] = dX[1][n];
      B[2][3 * n + 2] = dX[2][n];
      B[3][3 * n] = dX[1][n];
      B[3][3 * n + 1] = dX[0][n];
      B[4][3 * n + 1] = dX[2][n];
      B[4][3 * n + 2] = dX[1][n];
      B[5][3 * n] = dX[2][n];
      B[5][3 * n + 2] = dX[0][n];
    }
    double jac = det * 1.0;
    double BtD[24][6];
    for(int i = 0; i < 24; i++)
      for(int k = 0; k < 6; k++)
      {
        double s = 0.0;
        for(int l = 0; l < 6; l++)
          s += B[l][i] * D[6 * l + k];
        BtD[i][k] = s;
      }
    for(int i = 0; i < 24; i++)
      for(int j = 0; j < 24; j++)
      {
        double s = 0.0;
        for(int k = 0; k < 6; k++)
          s += BtD[i][k] * B[k][j];
        Ke[24 * i + j] += s * jac;
      }
    vol += jac;
  }
  if(volume)
    *volume = vol;
}

/* SIMP (src/problem/elasticity.hpp:13-17). */
static inline double or_simp(double e1, double e2, double rho, double p)
{
  return (1.0 - pow(rho, p)) * e1 + pow(rho, p) * e2;
}

/* ------------------------------------------------------------------------ */
/* 5. Problem: mesh + BC + CSR pattern of K_ff (free x free).                */
/* ------------------------------------------------------------------------ */
typedef struct
{
  int nx, ny, nz;
  double lx, ly, lz;
  int numnp, nelx, neq, numeq;
  double E1, E2, nu, pp;
  double *xyz;
  int *conn;
  int *dof, *has_dirich, *node_flag;
  double *node_dval; /* prescribed values, 0 on free components */
  double *fext;      /* numeq */
  double *fint;      /* numeq: K_fc u_c of the last assembly */
  double Ke0[576];
  double vol0;
  /* CSR of K_ff */
  long nnz;
  long *rowptr;
  int *col;
  double *val;
  double *diag;
  /* per node: position offsets of its 27 neighbour slots inside a row */
  int *slot_off; /* numnp*27, -1 if no neighbour / no free column */
  double *Ee;    /* nelx */
  int assembled;
} or_problem;

static void or_problem_free(or_problem *P)
{
  if(!P)
    return;
  free(P->xyz);
  free(P->conn);
  free(P->dof);
  free(P->has_dirich);
  free(P->node_flag);
  free(P->node_dval);
  free(P->fext);
  free(P->fint);
  free(P->rowptr);
  free(P->col);
  free(P->val);
  free(P->diag);
  free(P->slot_off);
  free(P->Ee);
  free(P);
}

void or_problem_destroy(or_problem *P) { or_problem_free(P); }

or_problem *or_problem_create(int nx, int ny, int nz, double lx, double ly,
                              double lz, double E1, double E2, double nu,
                              double pp, int ndir, const int *dflag,
                              const double *dval, const double *dbox,
                              int nload, const double *lval,
                              const double *lbox, int *status)
{
  *status = OR_OK;
  if(nx < 1 || ny < 1 || nz < 1)
  {
    *status = OR_ERR_ARG;
    return NULL;
  }
  or_problem *P = (or_problem *)calloc(1, sizeof(or_problem));
  P->nx = nx;
  P->ny = ny;
  P->nz = nz;
  P->lx = lx;
  P->ly = ly;
  P->lz = lz;
  P->E1 = E1;
  P->E2 = E2;
  P->nu = nu;
  P->pp = pp;
  const long NX = nx + 1, NY = ny + 1, NZ = nz + 1;
  P->numnp = (int)(NX * NY * NZ);
  P->nelx = nx * ny * nz;
  P->neq = 3 * P->numnp;
  P->xyz = (double *)malloc(sizeof(double) * 3 * P->numnp);
  P->conn = (int *)malloc(sizeof(int) * 8 * (long)P->nelx);
  or_mesh_box(nx, ny, nz, lx, ly, lz, P->xyz, P->conn);
  P->dof = (int *)malloc(sizeof(int) * 3 * P->numnp);
  P->has_dirich = (int *)malloc(sizeof(int) * P->numnp);
  P->node_flag = (int *)malloc(sizeof(int) * 3 * P->numnp);
  P->node_dval = (double *)malloc(sizeof(double) * 3 * P->numnp);
  P->numeq = or_count_dof(P->numnp, P->xyz, ndir, dflag, dval, dbox, P->dof,
                          P->has_dirich, P->node_flag, P->node_dval);
  /* only flagged components carry a prescribed value into the solve
     (LinearAnalysis::solve, src/analysis/linear.hpp:63-71) */
  for(long i = 0; i < 3L * P->numnp; i++)
    if(P->node_flag[i] != 1)
      P->node_dval[i] = 0.0;
  P->fext = (double *)calloc(P->numeq > 0 ? P->numeq : 1, sizeof(double));
  P->fint = (double *)calloc(P->numeq > 0 ? P->numeq : 1, sizeof(double));
  int st = or_point_loads(P->numnp, P->xyz, P->dof, P->numeq, P->nelx, P->conn, nload, lval,
                          lbox, P->fext);
  if(st != OR_OK)
  {
    *status = st;
    or_problem_free(P);
    return NULL;
  }
  /* Ke0 of the first element at E = 1 */
  double X[24];
  for(int a = 0; a < 8; a++)
    for(int c = 0; c < 3; c++)
      X[3 * a + c] = P->xyz[3 * P->conn[a] + c];
  or_hexa8_ke(X, 1.0, nu, P->Ke0, &P->vol0);

  /* CSR pattern: the row of free DOF (n, c) holds the free components of the
     27 neighbour nodes in ascending node id, i.e. ascending column. */
  P->rowptr = (long *)malloc(sizeof(long) * (P->numeq + 1));
  P->slot_off = (int *)malloc(sizeof(int) * 27 * (long)P->numnp);
  long nnz = 0;
  int row = 0;
  for(long k = 0; k < NZ; k++)
    for(long j = 0; j < NY; j++)
      for(long i = 0; i < NX; i++)
      {
        long n = i + j * NX + k * NX * NY;
        int len = 0;
        for(int s = 0; s < 27; s++)
        {
          int dx = s % 3 - 1, dy = (s / 3) % 3 - 1, dz = s / 9 - 1;
          long ii = i + dx, jj = j + dy, kk = k + dz;
          int *so = P->slot_off + 27 * n + s;
          *so = -1;
          if(ii < 0 || ii >= NX || jj < 0 || jj >= NY || kk < 0 || kk >= NZ)
            continue;
          long m = ii + jj * NX + kk * NX * NY;
          int nfree = 0;
          for(int c = 0; c < 3; c++)
            if(P->dof[3 * m + c] < P->numeq)
              nfree++;
          if(nfree)
            *so = len;
          len += nfree;
        }
        for(int c = 0; c < 3; c++)
          if(P->dof[3 * n + c] < P->numeq)
          {
            P->rowptr[row++] = nnz;
            nnz += len;
          }
      }
  P->rowptr[P->numeq] = nnz;
  P->nnz = nnz;
  P->col = (int *)malloc(sizeof(int) * (nnz > 0 ? nnz : 1));
  P->val = (double *)malloc(sizeof(double) * (nnz > 0 ? nnz : 1));
  P->diag = (double *)malloc(sizeof(double) * (P->numeq > 0 ? P->numeq : 1));
  P->Ee = (double *)malloc(sizeof(double) * P->nelx);
#pragma omp parallel for schedule(static)
  for(long n = 0; n < P->numnp; n++)
  {
    long i = n % NX, j = (n / NX) % NY, k = n / (NX * NY);
    for(int c = 0; c < 3; c++)
    {
      int r = P->dof[3 * n + c];
      if(r >= P->numeq)
        continue;
      long p = P->rowptr[r];
      for(int s = 0; s < 27; s++)
      {
        int dx = s % 3 - 1, dy = (s / 3) % 3 - 1, dz = s / 9 - 1;
        long ii = i + dx, jj = j + dy, kk = k + dz;
        if(ii < 0 || ii >= NX || jj < 0 || jj >= NY || kk < 0 || kk >= NZ)
          continue;
        long m = ii + jj * NX + kk * NX * NY;
        for(int d = 0; d < 3; d++)
          if(P->dof[3 * m + d] < P->numeq)
            P->col[p++] = P->dof[3 * m + d];
      }
    }
  }
  return P;
}

void or_problem_sizes(const or_problem *P, int *out)
{
  out[0] = P->numnp;
  out[1] = P->nelx;
  out[2] = P->neq;
  out[3] = P->numeq;
}
long or_problem_nnz(const or_problem *P) { return P->nnz; }
void or_problem_dof(const or_problem *P, int *dof)
{
  memcpy(dof, P->dof, sizeof(int) * 3 * P->numnp);
}
void or_problem_fext(const or_problem *P, double *f)
{
  memcpy(f, P->fext, sizeof(double) * P->numeq);
}
void or_problem_ke0(const or_problem *P, double *ke, double *vol)
{
  memcpy(ke, P->Ke0, sizeof(double) * 576);
  *vol = P->vol0;
}
void or_problem_xyz(const or_problem *P, double *xyz)
{
  memcpy(xyz, P->xyz, sizeof(double) * 3 * P->numnp);
}
void or_problem_conn(const or_problem *P, int *conn)
{
  memcpy(conn, P->conn, sizeof(int) * 8 * (long)P->nelx);
}
void or_problem_csr(const or_problem *P, long *rowptr, int *col, double *val)
{
  memcpy(rowptr, P->rowptr, sizeof(long) * (P->numeq + 1));
  memcpy(col, P->col, sizeof(int) * P->nnz);
  memcpy(val, P->val, sizeof(double) * P->nnz);
}

/* ------------------------------------------------------------------------ */
/* 6. Assembly: LinearAnalysis::assemblingK (src/analysis/linear.hpp:117-   */
/*    166) with LinearElastic::makeKeFint (elasticity.cpp:211-255) and       */
/*    assembling() (src/misc/assembling.hpp:19-39): Ke_e = E(rho_e) Ke0 added */
/*    at free x free positions; fint = fe restricted to free rows with the    */
/*    element displacement = prescribed values (node.val before the solve).  */
/* ------------------------------------------------------------------------ */
void or_assemble(or_problem *P, const double *design_s)
{
  const long NX = P->nx + 1, NY = P->ny + 1;
  const int nx = P->nx, ny = P->ny, nz = P->nz;
  for(long e = 0; e < P->nelx; e++)
    P->Ee[e] = or_simp(P->E1, P->E2, design_s[e], P->pp);
  memset(P->val, 0, sizeof(double) * P->nnz);
  memset(P->fint, 0, sizeof(double) * P->numeq);
  static const int lofs[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0},
                                 {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};
  /* 8 colours by element-index parity: elements of one colour share no node */
  for(int colour = 0; colour < 8; colour++)
  {
    int ci = colour & 1, cj = (colour >> 1) & 1, ck = (colour >> 2) & 1;
    int ni = (nx - ci + 1) / 2, nj = (ny - cj + 1) / 2, nk = (nz - ck + 1) / 2;
    long total = (long)ni * nj * nk;
#pragma omp parallel for schedule(static)
    for(long t = 0; t < total; t++)
    {
      long i = ci + 2 * (t % ni), j = cj + 2 * ((t / ni) % nj),
           k = ck + 2 * (t / ((long)ni * nj));
      long e = i + j * nx + k * (long)nx * ny;
      const int *cn = P->conn + 8 * e;
      double E = P->Ee[e];
      double Ke[576];
      for(int q = 0; q < 576; q++)
        Ke[q] = E * P->Ke0[q];
      for(int a = 0; a < 8; a++)
        for(int c = 0; c < 3; c++)
        {
          int r = P->dof[3 * cn[a] + c];
          if(r >= P->numeq)
            continue;
          long base = P->rowptr[r];
          double fe = 0.0;
          for(int b = 0; b < 8; b++)
          {
            int s = (lofs[b][0] - lofs[a][0] + 1) +
                    3 * (lofs[b][1] - lofs[a][1] + 1) +
                    9 * (lofs[b][2] - lofs[a][2] + 1);
            int so = P->slot_off[27 * (long)cn[a] + s];
            int pos = so;
            for(int d = 0; d < 3; d++)
            {
              double kv = Ke[24 * (3 * a + c) + 3 * b + d];
              fe += kv * P->node_dval[3 * cn[b] + d];
              if(P->dof[3 * cn[b] + d] < P->numeq)
                P->val[base + pos++] += kv;
            }
          }
          P->fint[r] += fe;
        }
    }
  }
  (void)NX;
  (void)NY;
#pragma omp parallel for schedule(static)
  for(long r = 0; r < P->numeq; r++)
  {
    double d = 0.0;
    for(long p = P->rowptr[r]; p < P->rowptr[r + 1]; p++)
      if(P->col[p] == r)
        d = P->val[p];
    P->diag[r] = d;
  }
  P->assembled = 1;
}

/* y = K_ff x (CSR, row order) */
void or_apply_K(const or_problem *P, const double *x, double *y)
{
#pragma omp parallel for schedule(static)
  for(long r = 0; r < P->numeq; r++)
  {
    double s = 0.0;
    for(long p = P->rowptr[r]; p < P->rowptr[r + 1]; p++)
      s += P->val[p] * x[P->col[p]];
    y[r] = s;
  }
}

static double or_dot(const double *a, const double *b, long n)
{
  double s = 0.0;
#pragma omp parallel for reduction(+ : s) schedule(static)
  for(long i = 0; i < n; i++)
    s += a[i] * b[i];
  return s;
}

/* ------------------------------------------------------------------------ */
/* 7. Jacobi-preconditioned CG: Solvers::ScalingCG (src/analysis/solver/     */
/*    CG.cpp:56-99), the hand-written equivalent of the "Eigen_CG" solver    */
/*    (solvers.cpp:63-91, DiagonalPreconditioner).  Zero initial guess; stop */
/*    after the iteration whose ||r|| < tol ||b||, or once iter > maxIter.   */
/* ------------------------------------------------------------------------ */
int or_pcg(const or_problem *P, const double *rhs, double *sol, double tol,
           int maxit, int *iters_out, double *relres_out)
{
  long n = P->numeq;
  double *r = (double *)malloc(sizeof(double) * (n ? n : 1));
  double *p = (double *)malloc(sizeof(double) * (n ? n : 1));
  double *z = (double *)malloc(sizeof(double) * (n ? n : 1));
  double *Ap = (double *)malloc(sizeof(double) * (n ? n : 1));
  for(long i = 0; i < n; i++)
  {
    sol[i] = 0.0;
    r[i] = rhs[i];
    p[i] = r[i] / P->diag[i];
    z[i] = p[i];
  }
  double bnorm = sqrt(or_dot(rhs, rhs, n));
  double zr = or_dot(z, r, n);
  double rnorm = bnorm;
  int iter = 0;
  while(1)
  {
    iter++;
    or_apply_K(P, p, Ap);
    double alpha = zr / or_dot(p, Ap, n);
#pragma omp parallel for schedule(static)
    for(long i = 0; i < n; i++)
    {
      sol[i] += alpha * p[i];
      r[i] -= alpha * Ap[i];
      z[i] = r[i] / P->diag[i];
    }
    double zr1 = or_dot(z, r, n);
    double beta = zr1 / zr;
#pragma omp parallel for schedule(static)
    for(long i = 0; i < n; i++)
      p[i] = beta * p[i] + z[i];
    zr = zr1;
    rnorm = sqrt(or_dot(r, r, n));
    if(rnorm < tol * bnorm)
      break;
    if(iter > maxit)
      break;
  }
  free(r);
  free(p);
  free(z);
  free(Ap);
  if(iters_out)
    *iters_out = iter;
  if(relres_out)
    *relres_out = bnorm > 0 ? rnorm / bnorm : 0.0;
  return OR_OK;
}

/* LinearAnalysis::solve (src/analysis/linear.hpp:55-104): assemble, fres =
   fext - fint, Jacobi-PCG.  Returns value.val (numeq). */
int or_linear_solve(or_problem *P, const double *design_s, double tol,
                    int maxit, double *val, int *iters, double *relres)
{
  or_assemble(P, design_s);
  double *fres = (double *)malloc(sizeof(double) * (P->numeq ? P->numeq : 1));
  for(long i = 0; i < P->numeq; i++)
    fres[i] = P->fext[i] - P->fint[i];
  int st = or_pcg(P, fres, val, tol, maxit, iters, relres);
  free(fres);
  return st;
}

/* divideValIntoNode (src/analysis/analysis_utility.hpp:9-31): free
   components from val, constrained ones from the prescribed value, and any
   |v| < 1e-15 set to 0. */
void or_node_values(const or_problem *P, const double *val, double *node_val)
{
#pragma omp parallel for schedule(static)
  for(long n = 0; n < P->numnp; n++)
    for(int c = 0; c < 3; c++)
    {
      int d = P->dof[3 * n + c];
      double v = (d >= P->numeq) ? P->node_dval[3 * n + c] : val[d];
      if(fabs(v) < 1.0e-15)
        v = 0.0;
      node_val[3 * n + c] = v;
    }
}

/* object_f = dis.val . force.fext (opt_macro_oc.cpp:110). */
double or_compliance(const or_problem *P, const double *val)
{
  double s = 0.0;
  for(long i = 0; i < P->numeq; i++)
    s += val[i] * P->fext[i];
  return s;
}

/* Driver sensitivity() (sample/algorithm/opt-macro-oc/opt_macro_oc.cpp:
   182-212; opt_macro_mma_nondesign.cpp:188-218):
   dfds = -(dE/E) u_e^T Ke_e u_e with Ke_e = E Ke0, dgds = volume * scale. */
void or_sensitivity(const or_problem *P, const double *design_s,
                    const double *node_val, double dgds_scale, double *dfds,
                    double *dgds)
{
#pragma omp parallel for schedule(static)
  for(long e = 0; e < P->nelx; e++)
  {
    double dens = design_s[e];
    double young = (1.0 - pow(dens, P->pp)) * P->E1 + pow(dens, P->pp) * P->E2;
    double dyoung = P->pp * pow(dens, P->pp - 1.0) * (P->E2 - P->E1);
    double Er = dyoung / young;
    double u[24];
    const int *cn = P->conn + 8 * e;
    for(int a = 0; a < 8; a++)
      for(int c = 0; c < 3; c++)
        u[3 * a + c] = node_val[3 * cn[a] + c];
    double q = 0.0;
    for(int i = 0; i < 24; i++)
    {
      double s = 0.0;
      for(int j = 0; j < 24; j++)
        s += (young * P->Ke0[24 * i + j]) * u[j];
      q += u[i] * s;
    }
    dfds[e] = -Er * q;
    dgds[e] = P->vol0 * dgds_scale;
  }
}

/* ------------------------------------------------------------------------ */
/* 8. Density filter: Filter<E,N> (src/optimization/filter.hpp).            */
/* ------------------------------------------------------------------------ */
typedef struct
{
  int n;
  double R;
  long *ptr;
  int *id;
  double *dis;
  double *aa; /* dfilters_ds: sum of weights of the last forward call */
  int have_forward;
} or_filter;

void or_filter_destroy(or_filter *F)
{
  if(!F)
    return;
  free(F->ptr);
  free(F->id);
  free(F->dis);
  free(F->aa);
  free(F);
}

/* Filter::preNeighbour (filter.hpp:254-297): centroid = sum_a x_a / ne in
   node order; neighbours j (ascending id) with |c_i - c_j| <= R. */
static void or_centroids(const or_problem *P, double *cen)
{
  for(long e = 0; e < P->nelx; e++)
  {
    const int *cn = P->conn + 8 * e;
    for(int d = 0; d < 3; d++)
    {
      double s = 0.0;
      for(int a = 0; a < 8; a++)
        s += P->xyz[3 * cn[a] + d] / 8;
      cen[3 * e + d] = s;
    }
  }
}

static double or_dist3(const double *a, const double *b)
{
  double dx = a[0] - b[0], dy = a[1] - b[1], dz = a[2] - b[2];
  return sqrt(dx * dx + dy * dy + dz * dz);
}

/* O(N^2) restatement, for any set of centroids (ndim 2 or 3 given as 3-vectors
   with a zero third coordinate). */
or_filter *or_filter_create_centroids(int n, const double *cen, double R)
{
  or_filter *F = (or_filter *)calloc(1, sizeof(or_filter));
  F->n = n;
  F->R = R;
  F->ptr = (long *)malloc(sizeof(long) * (n + 1));
  F->aa = (double *)calloc(n > 0 ? n : 1, sizeof(double));
  long cnt = 0;
  for(int i = 0; i < n; i++)
    for(int j = 0; j < n; j++)
      if(or_dist3(cen + 3 * i, cen + 3 * j) <= R)
        cnt++;
  F->id = (int *)malloc(sizeof(int) * (cnt ? cnt : 1));
  F->dis = (double *)malloc(sizeof(double) * (cnt ? cnt : 1));
  long p = 0;
  for(int i = 0; i < n; i++)
  {
    F->ptr[i] = p;
    for(int j = 0; j < n; j++)
    {
      double d = or_dist3(cen + 3 * i, cen + 3 * j);
      if(d <= R)
      {
        F->id[p] = j;
        F->dis[p] = d;
        p++;
      }
    }
  }
  F->ptr[n] = p;
  return F;
}

/* Same lists, same order, found by scanning only the index box of +-(ceil
   (R/h)+1) elements around i in ascending element id. */
or_filter *or_filter_create(const or_problem *P, double R, int faithful)
{
  long n = P->nelx;
  double *cen = (double *)malloc(sizeof(double) * 3 * n);
  or_centroids(P, cen);
  if(faithful)
  {
    or_filter *F = or_filter_create_centroids((int)n, cen, R);
    free(cen);
    return F;
  }
  const int nx = P->nx, ny = P->ny, nz = P->nz;
  double hx = P->lx / nx, hy = P->ly / ny, hz = P->lz / nz;
  int rx = (int)ceil(R / hx) + 1, ry = (int)ceil(R / hy) + 1,
      rz = (int)ceil(R / hz) + 1;
  or_filter *F = (or_filter *)calloc(1, sizeof(or_filter));
  F->n = (int)n;
  F->R = R;
  F->ptr = (long *)malloc(sizeof(long) * (n + 1));
  F->aa = (double *)calloc(n, sizeof(double));
  int *cnt = (int *)malloc(sizeof(int) * n);
#pragma omp parallel for schedule(static)
  for(long e = 0; e < n; e++)
  {
    int i = (int)(e % nx), j = (int)((e / nx) % ny), k = (int)(e / ((long)nx * ny));
    int c = 0;
    for(int kk = k - rz; kk <= k + rz; kk++)
      for(int jj = j - ry; jj <= j + ry; jj++)
        for(int ii = i - rx; ii <= i + rx; ii++)
        {
          if(ii < 0 || ii >= nx || jj < 0 || jj >= ny || kk < 0 || kk >= nz)
            continue;
          long f = ii + (long)jj * nx + (long)kk * nx * ny;
          if(or_dist3(cen + 3 * e, cen + 3 * f) <= R)
            c++;
        }
    cnt[e] = c;
  }
  long p = 0;
  for(long e = 0; e < n; e++)
  {
    F->ptr[e] = p;
    p += cnt[e];
  }
  F->ptr[n] = p;
  F->id = (int *)malloc(sizeof(int) * (p ? p : 1));
  F->dis = (double *)malloc(sizeof(double) * (p ? p : 1));
#pragma omp parallel for schedule(static)
  for(long e = 0; e < n; e++)
  {
    int i = (int)(e % nx), j = (int)((e / nx) % ny), k = (int)(e / ((long)nx * ny));
    long q = F->ptr[e];
    for(int kk = k - rz; kk <= k + rz; kk++)
      for(int jj = j - ry; jj <= j + ry; jj++)
        for(int ii = i - rx; ii <= i + rx; ii++)
        {
          if(ii < 0 || ii >= nx || jj < 0 || jj >= ny || kk < 0 || kk >= nz)
            continue;
          long f = ii + (long)jj * nx + (long)kk * nx * ny;
          double d = or_dist3(cen + 3 * e, cen + 3 * f);
          if(d <= R)
          {
            F->id[q] = (int)f;
            F->dis[q] = d;
            q++;
          }
        }
  }
  free(cnt);
  free(cen);
  return F;
}

long or_filter_nnz(const or_filter *F) { return F->ptr[F->n]; }
void or_filter_lists(const or_filter *F, long *ptr, int *id, double *dis)
{
  memcpy(ptr, F->ptr, sizeof(long) * (F->n + 1));
  memcpy(id, F->id, sizeof(int) * F->ptr[F->n]);
  memcpy(dis, F->dis, sizeof(double) * F->ptr[F->n]);
}

/* Filter::densityFilter (filter.hpp:107-155).  Forward: out_i =
   sum_j (R - d_ij) in_j / sum_j (R - d_ij), caching a_i = sum_j w_ij and
   failing when a_i < 1e-10.  Transposed (is_sens): out_i =
   sum_j w_ij in_j / a_j using the a_j of the last forward call. */
int or_filter_density(or_filter *F, const double *in, double *out, int is_sens)
{
  int n = F->n;
  int bad = 0;
  if(!is_sens)
  {
#pragma omp parallel for schedule(static) reduction(| : bad)
    for(int i = 0; i < n; i++)
    {
      double aa = 0.0, bb = 0.0;
      for(long p = F->ptr[i]; p < F->ptr[i + 1]; p++)
      {
        double w = F->R - F->dis[p];
        aa += w;
        bb += w * in[F->id[p]];
      }
      if(aa < 1.0e-10)
        bad = 1;
      out[i] = bb / aa;
      F->aa[i] = aa;
    }
    if(bad)
      return OR_ERR_FILTER;
    F->have_forward = 1;
  }
  else
  {
    if(!F->have_forward)
      return OR_ERR_STATE;
#pragma omp parallel for schedule(static)
    for(int i = 0; i < n; i++)
    {
      double s = 0.0;
      for(long p = F->ptr[i]; p < F->ptr[i + 1]; p++)
      {
        double w = F->R - F->dis[p];
        s += w * in[F->id[p]] / F->aa[F->id[p]];
      }
      out[i] = s;
    }
  }
  return OR_OK;
}

/* Filter::sensitivityFilter (filter.hpp:77-104). */
void or_filter_sensitivity(const or_filter *F, const double *design_s,
                           const double *dfds, const double *volume,
                           double *out)
{
#pragma omp parallel for schedule(static)
  for(int i = 0; i < F->n; i++)
  {
    double aa = 0.0, bb = 0.0;
    for(long p = F->ptr[i]; p < F->ptr[i + 1]; p++)
    {
      int j = F->id[p];
      double w = F->R - F->dis[p];
      aa += w;
      bb += (w * design_s[j] * dfds[j]) / (design_s[j] * volume[j]);
    }
    double cc = (design_s[i] * volume[i]) / (design_s[i] * aa);
    out[i] = cc * bb;
  }
}

/* Filter::threshold / thresholdDerivative (filter.hpp:217-249). */
void or_threshold(int n, const double *in, double beta, double T, double *out)
{
  for(int i = 0; i < n; i++)
    out[i] = 0.5 * (tanh(T * beta) + tanh(beta * (in[i] - T))) / tanh(T * beta);
}
void or_threshold_deriv(int n, const double *in, double beta, double T,
                        double *out)
{
  for(int i = 0; i < n; i++)
    out[i] = (0.5 * (beta * (1.0 - pow(tanh(beta * (in[i] - T)), 2.0))) /
              tanh(T * beta));
}

/* ------------------------------------------------------------------------ */
/* 9. OC::UpdateVariables (src/optimization/opt-solver/OCSolver.hpp:21-79). */
/*    Bisection on lambda in [lmin, lmax] while (l1-l0)/(l1+l0) > eps and    */
/*    counter < maxiter; x+ = x * max(0, -dfdx/(dgdx lambda))^iota clamped    */
/*    to [max(xmin,(1-m)x), min(xmax,(1+m)x)]; lambda0 = lambda when          */
/*    g(x+) - g > 0.  x takes the last trial.                                */
/* ------------------------------------------------------------------------ */
typedef double (*or_volume_fn)(const double *x, void *user);

typedef struct
{
  double move, iota, lmin, lmax, leps;
  int maxiter;
} or_oc_params;

int or_oc_update(int n, double *x, const double *dfdx, double g,
                 const double *dgdx, const double *xmin, const double *xmax,
                 const or_oc_params *prm, or_volume_fn gfun, void *user,
                 int *steps_out)
{
  double l0 = prm->lmin, l1 = prm->lmax, lambda;
  /* xkp1 starts as zeros and is assigned to x even when no step ran */
  double *xk = (double *)calloc(n ? n : 1, sizeof(double));
  int counter = 0;
  while((l1 - l0) / (l1 + l0) > prm->leps && prm->maxiter > counter)
  {
    lambda = 0.5 * (l1 + l0);
#pragma omp parallel for schedule(static)
    for(int i = 0; i < n; i++)
    {
      double v = -dfdx[i] / (dgdx[i] * lambda);
      double xn = pow(v > 0.0 ? v : 0.0, prm->iota) * x[i];
      double lo = (1.0 - prm->move) * x[i];
      double hi = (1.0 + prm->move) * x[i];
      lo = xmin[i] > lo ? xmin[i] : lo;
      hi = xmax[i] < hi ? xmax[i] : hi;
      if(xn < lo)
        xn = lo;
      else if(xn > hi)
        xn = hi;
      xk[i] = xn;
    }
    if(gfun(xk, user) - g > 0.0)
      l0 = lambda;
    else
      l1 = lambda;
    counter++;
  }
  memcpy(x, xk, sizeof(double) * n);
  free(xk);
  if(steps_out)
    *steps_out = counter;
  return counter >= prm->maxiter ? 1 : OR_OK;
}

int or_helmholtz_filter(int nx, int ny, int nz, double lx, double ly, double lz, double R,
                        const double *in, double *out, int sens, double tol, int maxit,
                        int *iters_out);

/* Volume functor of the sample drivers (opt_macro_oc.cpp:153-164):
   g(x) = sum_i thr(filter(x))_i v_i, with the radius filter F or, when
   helm_R > 0, the Helmholtz filter of the box (nx, ny, nz, lx, ly, lz). */
typedef struct
{
  or_filter *F;
  int use_threshold;
  double beta, T;
  const double *vol;
  double *tmp, *tmp2;
  int n;
  double helm_R, helm_tol;
  int nx, ny, nz;
  double lx, ly, lz;
} or_filter_volume;

static double or_filter_volume_fn(const double *x, void *user)
{
  or_filter_volume *fv = (or_filter_volume *)user;
  int n = fv->n;
  if(fv->helm_R > 0.0)
    or_helmholtz_filter(fv->nx, fv->ny, fv->nz, fv->lx, fv->ly, fv->lz, fv->helm_R, x,
                        fv->tmp, 0, fv->helm_tol, 10000, NULL);
  else
    or_filter_density(fv->F, x, fv->tmp, 0);
  const double *t = fv->tmp;
  if(fv->use_threshold)
  {
    or_threshold(n, fv->tmp, fv->beta, fv->T, fv->tmp2);
    t = fv->tmp2;
  }
  double g = 0.0;
  for(int i = 0; i < n; i++)
    g += t[i] * fv->vol[i];
  return g;
}

/* ------------------------------------------------------------------------ */
/* 10. MMA (Svanberg; src/optimization/opt-solver/MMASolver.cpp, after      */
/*     Aage/Dumas, MIT).  State and steps follow MMASolver::Update (:66-82):  */
/*     GenSub (:400-512), then the dual interior-point method SolveDIP       */
/*     (:88-154) with XYZofLAMBDA (:359-398), DualGrad (:346-357), DualHess   */
/*     (:238-344), DualLineSearch (:214-236), DualResidual (:184-212) and    */
/*     the dense LU Factorize/Solve (:514-553) for m > 1.                    */
/* ------------------------------------------------------------------------ */
typedef struct
{
  int n, m, iter;
  double xmamieps, epsimin, raa0, move, albefa, asyminit, asymdec, asyminc;
  double *a, *c, *d, *y, *lam, *mu, *s;
  double z;
  double *low, *upp, *alpha, *beta, *p0, *q0, *pij, *qij, *b, *grad, *hess;
  double *xold1, *xold2;
  int last_outloop, last_inner_total;
} or_mma;

or_mma *or_mma_create(int n, int m, double a, double c, double d)
{
  or_mma *M = (or_mma *)calloc(1, sizeof(or_mma));
  M->n = n;
  M->m = m;
  M->iter = 0;
  M->xmamieps = 1.0e-5;
  M->epsimin = sqrt((double)(n + m)) * 1e-9;
  M->raa0 = 0.00001;
  M->move = 0.15;
  M->albefa = 0.2;
  M->asyminit = 0.2;
  M->asymdec = 0.7;
  M->asyminc = 1.2;
#define OR_ALLOC(p, k) p = (double *)calloc((k) > 0 ? (k) : 1, sizeof(double))
  OR_ALLOC(M->a, m);
  OR_ALLOC(M->c, m);
  OR_ALLOC(M->d, m);
  OR_ALLOC(M->y, m);
  OR_ALLOC(M->lam, m);
  OR_ALLOC(M->mu, m);
  OR_ALLOC(M->s, 2 * m);
  OR_ALLOC(M->low, n);
  OR_ALLOC(M->upp, n);
  OR_ALLOC(M->alpha, n);
  OR_ALLOC(M->beta, n);
  OR_ALLOC(M->p0, n);
  OR_ALLOC(M->q0, n);
  OR_ALLOC(M->pij, (long)n * m);
  OR_ALLOC(M->qij, (long)n * m);
  OR_ALLOC(M->b, m);
  OR_ALLOC(M->grad, m);
  OR_ALLOC(M->hess, m * m);
  OR_ALLOC(M->xold1, n);
  OR_ALLOC(M->xold2, n);
#undef OR_ALLOC
  for(int j = 0; j < m; j++)
  {
    M->a[j] = a;
    M->c[j] = c;
    M->d[j] = d;
  }
  return M;
}

void or_mma_destroy(or_mma *M)
{
  if(!M)
    return;
  free(M->a);
  free(M->c);
  free(M->d);
  free(M->y);
  free(M->lam);
  free(M->mu);
  free(M->s);
  free(M->low);
  free(M->upp);
  free(M->alpha);
  free(M->beta);
  free(M->p0);
  free(M->q0);
  free(M->pij);
  free(M->qij);
  free(M->b);
  free(M->grad);
  free(M->hess);
  free(M->xold1);
  free(M->xold2);
  free(M);
}

void or_mma_set_move(or_mma *M, double mv) { M->move = mv; }
void or_mma_set_asymptotes(or_mma *M, double init, double dec, double inc)
{
  M->asyminit = init;
  M->asymdec = dec;
  M->asyminc = inc;
}
void or_mma_set_oscillation(or_mma *M, double a) { M->albefa = a; }
int or_mma_outloops(const or_mma *M) { return M->last_outloop; }
int or_mma_inner_total(const or_mma *M) { return M->last_inner_total; }
void or_mma_state(const or_mma *M, double *low, double *upp, double *xold1,
                  double *xold2)
{
  memcpy(low, M->low, sizeof(double) * M->n);
  memcpy(upp, M->upp, sizeof(double) * M->n);
  memcpy(xold1, M->xold1, sizeof(double) * M->n);
  memcpy(xold2, M->xold2, sizeof(double) * M->n);
}

static inline double or_max(double a, double b) { return a > b ? a : b; }
static inline double or_min(double a, double b) { return a < b ? a : b; }

static void or_mma_gensub(or_mma *M, const double *xval, const double *dfdx,
                          const double *gx, const double *dgdx,
                          const double *xmin, const double *xmax)
{
  const int n = M->n, m = M->m;
  M->iter++;
  if(M->iter < 3)
  {
    for(int i = 0; i < n; i++)
    {
      M->low[i] = xval[i] - M->asyminit * (xmax[i] - xmin[i]);
      M->upp[i] = xval[i] + M->asyminit * (xmax[i] - xmin[i]);
    }
  }
  else
  {
    for(int i = 0; i < n; i++)
    {
      double zzz = (xval[i] - M->xold1[i]) * (M->xold1[i] - M->xold2[i]);
      double gamma = zzz < 0.0 ? M->asymdec : (zzz > 0.0 ? M->asyminc : 1.0);
      M->low[i] = xval[i] - gamma * (M->xold1[i] - M->low[i]);
      M->upp[i] = xval[i] + gamma * (M->upp[i] - M->xold1[i]);
      double xmami = or_max(M->xmamieps, xmax[i] - xmin[i]);
      M->low[i] = or_max(M->low[i], xval[i] - 100.0 * xmami);
      M->low[i] = or_min(M->low[i], xval[i] - 1.0e-5 * xmami);
      M->upp[i] = or_max(M->upp[i], xval[i] + 1.0e-5 * xmami);
      M->upp[i] = or_min(M->upp[i], xval[i] + 100.0 * xmami);
      double xmi = xmin[i] - 1.0e-6;
      double xma = xmax[i] + 1.0e-6;
      if(xval[i] < xmi)
      {
        M->low[i] = xval[i] - (xma - xval[i]) / 0.9;
        M->upp[i] = xval[i] + (xma - xval[i]) / 0.9;
      }
      if(xval[i] > xma)
      {
        M->low[i] = xval[i] - (xval[i] - xmi) / 0.9;
        M->upp[i] = xval[i] + (xval[i] - xmi) / 0.9;
      }
    }
  }
  for(int i = 0; i < n; i++)
  {
    double al = or_max(xmin[i], M->low[i] + M->albefa * (xval[i] - M->low[i]));
    al = or_max(al, xval[i] - M->move * (xmax[i] - xmin[i]));
    M->alpha[i] = or_min(al, xmax[i]);
    double be = or_min(xmax[i], M->upp[i] - M->albefa * (M->upp[i] - xval[i]));
    be = or_min(be, xval[i] + M->move * (xmax[i] - xmin[i]));
    M->beta[i] = or_max(be, xmin[i]);
    double ux = M->upp[i] - xval[i], xl = xval[i] - M->low[i];
    double xmamiinv = 1.0 / or_max(M->xmamieps, xmax[i] - xmin[i]);
    double pq = 0.001 * fabs(dfdx[i]) + M->raa0 * xmamiinv;
    M->p0[i] = pow(ux, 2.0) * (or_max(0.0, dfdx[i]) + pq);
    M->q0[i] = pow(xl, 2.0) * (or_max(0.0, -1.0 * dfdx[i]) + pq);
    for(int j = 0; j < m; j++)
    {
      double gd = dgdx[(long)i * m + j];
      double pqj = 0.001 * fabs(gd) + M->raa0 * xmamiinv;
      M->pij[(long)i * m + j] = pow(ux, 2.0) * (or_max(0.0, gd) + pqj);
      M->qij[(long)i * m + j] = pow(xl, 2.0) * (or_max(0.0, -1.0 * gd) + pqj);
    }
  }
  for(int j = 0; j < m; j++)
  {
    double bj = -gx[j];
    for(int i = 0; i < n; i++)
      bj += M->pij[(long)i * m + j] / (M->upp[i] - xval[i]) +
            M->qij[(long)i * m + j] / (xval[i] - M->low[i]);
    M->b[j] = bj;
  }
}

static void or_mma_xyz(or_mma *M, double *x)
{
  const int n = M->n, m = M->m;
  double lamai = 0.0;
  for(int j = 0; j < m; j++)
  {
    if(M->lam[j] < 0.0)
      M->lam[j] = 0;
    M->y[j] = or_max(0.0, M->lam[j] - M->c[j]);
    lamai += M->lam[j] * M->a[j];
  }
  M->z = or_max(0.0, 10.0 * (lamai - 1.0));
#pragma omp parallel for schedule(static)
  for(int i = 0; i < n; i++)
  {
    double pl = M->p0[i], ql = M->q0[i];
    for(int j = 0; j < m; j++)
    {
      pl += M->pij[(long)i * m + j] * M->lam[j];
      ql += M->qij[(long)i * m + j] * M->lam[j];
    }
    double xi = (sqrt(pl) * M->low[i] + sqrt(ql) * M->upp[i]) / (sqrt(pl) + sqrt(ql));
    if(xi < M->alpha[i])
      xi = M->alpha[i];
    if(xi > M->beta[i])
      xi = M->beta[i];
    x[i] = xi;
  }
}

static void or_mma_grad(or_mma *M, const double *x)
{
  const int n = M->n, m = M->m;
  for(int j = 0; j < m; j++)
  {
    double g = -M->b[j] - M->a[j] * M->z - M->y[j];
    for(int i = 0; i < n; i++)
      g += M->pij[(long)i * m + j] / (M->upp[i] - x[i]) +
           M->qij[(long)i * m + j] / (x[i] - M->low[i]);
    M->grad[j] = g;
  }
}

static void or_mma_hess(or_mma *M, const double *x)
{
  const int n = M->n, m = M->m;
  double *df2 = (double *)malloc(sizeof(double) * n);
  double *PQ = (double *)malloc(sizeof(double) * (long)n * m);
#pragma omp parallel for schedule(static)
  for(int i = 0; i < n; i++)
  {
    double pl = M->p0[i], ql = M->q0[i];
    for(int j = 0; j < m; j++)
    {
      pl += M->pij[(long)i * m + j] * M->lam[j];
      ql += M->qij[(long)i * m + j] * M->lam[j];
      PQ[(long)i * m + j] = M->pij[(long)i * m + j] / pow(M->upp[i] - x[i], 2.0) -
                            M->qij[(long)i * m + j] / pow(x[i] - M->low[i], 2.0);
    }
    df2[i] = -1.0 / (2.0 * pl / pow(M->upp[i] - x[i], 3.0) +
                     2.0 * ql / pow(x[i] - M->low[i], 3.0));
    double xp = (sqrt(pl) * M->low[i] + sqrt(ql) * M->upp[i]) / (sqrt(pl) + sqrt(ql));
    if(xp < M->alpha[i])
      df2[i] = 0.0;
    if(xp > M->beta[i])
      df2[i] = 0.0;
  }
  for(int i = 0; i < m; i++)
    for(int j = 0; j < m; j++)
    {
      double h = 0.0;
      for(int k = 0; k < n; k++)
        h += (0.0 + PQ[(long)k * m + i] * df2[k]) * PQ[(long)k * m + j];
      M->hess[i * m + j] = h;
    }
  double lamai = 0.0;
  for(int j = 0; j < m; j++)
  {
    if(M->lam[j] < 0.0)
      M->lam[j] = 0.0;
    lamai += M->lam[j] * M->a[j];
    if(M->lam[j] > M->c[j])
      M->hess[j * m + j] += -1.0;
    M->hess[j * m + j] += -M->mu[j] / M->lam[j];
  }
  if(lamai > 0.0)
    for(int j = 0; j < m; j++)
      for(int k = 0; k < m; k++)
        M->hess[j * m + k] += -10.0 * M->a[j] * M->a[k];
  double tr = 0.0;
  for(int i = 0; i < m; i++)
    tr += M->hess[i * m + i];
  double corr = 1e-4 * tr / m;
  if(-1.0 * corr < 1.0e-7)
    corr = -1.0e-7;
  for(int i = 0; i < m; i++)
    M->hess[i * m + i] += corr;
  free(df2);
  free(PQ);
}

static double or_mma_residual(or_mma *M, const double *x, double epsi)
{
  const int n = M->n, m = M->m;
  double nr = 0.0;
  for(int j = 0; j < m; j++)
  {
    double r = -M->b[j] - M->a[j] * M->z - M->y[j] + M->mu[j];
    double r2 = M->mu[j] * M->lam[j] - epsi;
    for(int i = 0; i < n; i++)
      r += M->pij[(long)i * m + j] / (M->upp[i] - x[i]) +
           M->qij[(long)i * m + j] / (x[i] - M->low[i]);
    if(nr < fabs(r))
      nr = fabs(r);
    if(nr < fabs(r2))
      nr = fabs(r2);
  }
  return nr;
}

static void or_mma_linesearch(or_mma *M)
{
  const int m = M->m;
  double theta = 1.005;
  for(int i = 0; i < m; i++)
  {
    if(theta < -1.01 * M->s[i] / M->lam[i])
      theta = -1.01 * M->s[i] / M->lam[i];
    if(theta < -1.01 * M->s[i + m] / M->mu[i])
      theta = -1.01 * M->s[i + m] / M->mu[i];
  }
  theta = 1.0 / theta;
  for(int i = 0; i < m; i++)
  {
    M->lam[i] = M->lam[i] + theta * M->s[i];
    M->mu[i] = M->mu[i] + theta * M->s[i + m];
  }
}

/* in-place LU without pivoting and the two triangular sweeps
   (MMASolver.cpp:514-553) */
static void or_lu(double *K, int n)
{
  for(int s = 0; s < n - 1; s++)
    for(int i = s + 1; i < n; i++)
    {
      K[i * n + s] = K[i * n + s] / K[s * n + s];
      for(int j = s + 1; j < n; j++)
        K[i * n + j] = K[i * n + j] - K[i * n + s] * K[s * n + j];
    }
}
static void or_lu_solve(const double *K, double *x, int n)
{
  for(int i = 1; i < n; i++)
  {
    double a = 0.0;
    for(int j = 0; j < i; j++)
      a = a - K[i * n + j] * x[j];
    x[i] = x[i] + a;
  }
  x[n - 1] = x[n - 1] / K[(n - 1) * n + (n - 1)];
  for(int i = n - 2; i >= 0; i--)
  {
    double a = x[i];
    for(int j = i + 1; j < n; j++)
      a = a - K[i * n + j] * x[j];
    x[i] = a / K[i * n + i];
  }
}

static void or_mma_dip(or_mma *M, double *x)
{
  const int m = M->m;
  for(int j = 0; j < m; j++)
  {
    M->lam[j] = M->c[j] / 2.0;
    M->mu[j] = 1.0;
  }
  const double tol = M->epsimin;
  double epsi = 1.0, err = 1.0;
  int outloop = 0, total = 0;
  while(epsi > tol && outloop < 100)
  {
    outloop++;
    int loop = 0;
    while(err > 0.9 * epsi && loop < 100)
    {
      loop++;
      total++;
      or_mma_xyz(M, x);
      or_mma_grad(M, x);
      for(int j = 0; j < m; j++)
        M->grad[j] = -1.0 * M->grad[j] - epsi / M->lam[j];
      or_mma_hess(M, x);
      if(m > 1)
      {
        or_lu(M->hess, m);
        or_lu_solve(M->hess, M->grad, m);
        for(int j = 0; j < m; j++)
          M->s[j] = M->grad[j];
      }
      else if(m > 0)
        M->s[0] = M->grad[0] / M->hess[0];
      for(int i = 0; i < m; i++)
        M->s[m + i] = -M->mu[i] + epsi / M->lam[i] - M->s[i] * M->mu[i] / M->lam[i];
      or_mma_linesearch(M);
      or_mma_xyz(M, x);
      err = or_mma_residual(M, x, epsi);
    }
    epsi = epsi * 0.1;
  }
  M->last_outloop = outloop;
  M->last_inner_total = total;
}

void or_mma_update(or_mma *M, double *xval, const double *dfdx,
                   const double *gx, const double *dgdx, const double *xmin,
                   const double *xmax)
{
  or_mma_gensub(M, xval, dfdx, gx, dgdx, xmin, xmax);
  memcpy(M->xold2, M->xold1, sizeof(double) * M->n);
  memcpy(M->xold1, xval, sizeof(double) * M->n);
  or_mma_dip(M, xval);
}

/* ------------------------------------------------------------------------ */
/* 11. One design iteration of the sample drivers:                          */
/*     sample/algorithm/opt-macro-oc/opt_macro_oc.cpp:83-172 (OC) and        */
/*     sample/algorithm/opt-macro-mma-nondesign/opt_macro_mma_nondesign.cpp: */
/*     90-178 (MMA), with the radius Filter and an optional threshold (the   */
/*     drivers always apply it with beta = min(2^(step/40), 16), T = 0.5).   */
/*     or_loop_set_helmholtz switches to the Helmholtz filter of             */
/*     opt_macro_oc.cpp:73-74 / opt_mma_Helmholtz.cpp:70-72 (solved to tol,   */
/*     the "Eigen_CG" default being 1e-10), also inside the OC functor.       */
/* ------------------------------------------------------------------------ */
typedef struct
{
  or_problem *P;
  or_filter *F;
  or_mma *M;
  int method; /* 0 = OC, 1 = MMA */
  int use_threshold;
  double T;
  double cg_tol;
  int cg_maxit;
  or_oc_params oc;
  int optstep;
  double V0;
  double *x, *xfil, *xthr, *thrd, *dfds, *dgds, *val, *node_val, *xmin, *xmax,
      *vol, *tmp, *tmp2;
  double compliance, constraint;
  int cg_iters, oc_steps, mma_outloops;
  double cg_relres;
  double t_filter, t_solve, t_sens, t_update, t_pcg;
  double helm_R, helm_tol; /* helm_R > 0: Helmholtz filter */
} or_loop;

void or_loop_set_helmholtz(or_loop *L, double R, double tol)
{
  L->helm_R = R;
  L->helm_tol = tol;
}

static int or_loop_filter(or_loop *L, const double *in, double *out, int sens)
{
  const or_problem *P = L->P;
  if(L->helm_R > 0.0)
  {
    int st = or_helmholtz_filter(P->nx, P->ny, P->nz, P->lx, P->ly, P->lz, L->helm_R, in,
                                 out, sens, L->helm_tol, 10000, NULL);
    return st == OR_OK ? OR_OK : st;
  }
  return or_filter_density(L->F, in, out, sens);
}

or_loop *or_loop_create(or_problem *P, or_filter *F, int method,
                        int use_threshold, double move, double xmin,
                        double xmax, double cg_tol, int cg_maxit,
                        const double *x0)
{
  or_loop *L = (or_loop *)calloc(1, sizeof(or_loop));
  long n = P->nelx;
  L->P = P;
  L->F = F;
  L->method = method;
  L->use_threshold = use_threshold;
  L->T = 0.5;
  L->cg_tol = cg_tol;
  L->cg_maxit = cg_maxit;
  L->oc.move = move;
  L->oc.iota = 0.5;
  L->oc.lmin = 0.0;
  L->oc.lmax = 1.0e4;
  L->oc.leps = 1.0e-5;
  L->oc.maxiter = 100;
  if(method == 1)
  {
    L->M = or_mma_create((int)n, 1, 0.0, 100000.0, 0.0);
    or_mma_set_move(L->M, move);
  }
#define OR_VEC(p) p = (double *)calloc(n, sizeof(double))
  OR_VEC(L->x);
  OR_VEC(L->xfil);
  OR_VEC(L->xthr);
  OR_VEC(L->thrd);
  OR_VEC(L->dfds);
  OR_VEC(L->dgds);
  OR_VEC(L->xmin);
  OR_VEC(L->xmax);
  OR_VEC(L->vol);
  OR_VEC(L->tmp);
  OR_VEC(L->tmp2);
#undef OR_VEC
  L->val = (double *)calloc(P->numeq ? P->numeq : 1, sizeof(double));
  L->node_val = (double *)calloc(3 * (long)P->numnp, sizeof(double));
  for(long e = 0; e < n; e++)
  {
    L->x[e] = x0[e];
    L->xmin[e] = xmin;
    L->xmax[e] = xmax;
    L->vol[e] = P->vol0;
  }
  return L;
}

void or_loop_destroy(or_loop *L)
{
  if(!L)
    return;
  or_mma_destroy(L->M);
  free(L->x);
  free(L->xfil);
  free(L->xthr);
  free(L->thrd);
  free(L->dfds);
  free(L->dgds);
  free(L->xmin);
  free(L->xmax);
  free(L->vol);
  free(L->tmp);
  free(L->tmp2);
  free(L->val);
  free(L->node_val);
  free(L);
}

int or_loop_step(or_loop *L)
{
  or_problem *P = L->P;
  const int n = P->nelx;
  double t0 = or_now();
  L->optstep++;
  int st = or_loop_filter(L, L->x, L->xfil, 0);
  if(st != OR_OK)
    return st;
  double beta = pow(2, (int)(L->optstep / 40));
  if(beta > 16.0)
    beta = 16.0;
  if(L->use_threshold)
  {
    or_threshold(n, L->xfil, beta, L->T, L->xthr);
    or_threshold_deriv(n, L->xfil, beta, L->T, L->thrd);
  }
  else
    for(int e = 0; e < n; e++)
    {
      L->xthr[e] = L->xfil[e];
      L->thrd[e] = 1.0;
    }
  double t1 = or_now();
  /* LinearAnalysis::solve = assemble, fres = fext - fint, PCG */
  or_assemble(P, L->xthr);
  double *rhs = (double *)malloc(sizeof(double) * (P->numeq ? P->numeq : 1));
  for(long i = 0; i < P->numeq; i++)
    rhs[i] = P->fext[i] - P->fint[i];
  double tp0 = or_now();
  or_pcg(P, rhs, L->val, L->cg_tol, L->cg_maxit, &L->cg_iters, &L->cg_relres);
  L->t_pcg += or_now() - tp0;
  free(rhs);
  or_node_values(P, L->val, L->node_val);
  double t2 = or_now();
  L->compliance = or_compliance(P, L->val);
  if(L->optstep == 1)
  {
    double V0 = 0.0;
    for(int e = 0; e < n; e++)
      V0 += L->xthr[e] * L->vol[e];
    L->V0 = V0;
    L->constraint = (L->method == 1) ? 0.0 : V0;
  }
  else
  {
    double g = 0.0;
    if(L->method == 1)
    {
      for(int e = 0; e < n; e++)
        g += L->xthr[e] * L->vol[e] / L->V0;
      g += -1.0;
    }
    else
      for(int e = 0; e < n; e++)
        g += L->xthr[e] * L->vol[e];
    L->constraint = g;
  }
  or_sensitivity(P, L->xthr, L->node_val, L->method == 1 ? 1.0 / L->V0 : 1.0,
                 L->dfds, L->dgds);
  for(int e = 0; e < n; e++)
  {
    L->dfds[e] *= L->thrd[e];
    L->dgds[e] *= L->thrd[e];
  }
  or_loop_filter(L, L->dfds, L->tmp, 1);
  memcpy(L->dfds, L->tmp, sizeof(double) * n);
  or_loop_filter(L, L->dgds, L->tmp, 1);
  memcpy(L->dgds, L->tmp, sizeof(double) * n);
  double t3 = or_now();
  if(L->method == 1)
  {
    double g = L->constraint;
    or_mma_update(L->M, L->x, L->dfds, &g, L->dgds, L->xmin, L->xmax);
    L->mma_outloops = L->M->last_outloop;
  }
  else
  {
    or_filter_volume fv = {L->F, L->use_threshold, beta, L->T, L->vol, L->tmp, L->tmp2,
                           n, L->helm_R, L->helm_tol, P->nx, P->ny, P->nz, P->lx, P->ly,
                           P->lz};
    or_oc_update(n, L->x, L->dfds, L->V0, L->dgds, L->xmin, L->xmax, &L->oc,
                 or_filter_volume_fn, &fv, &L->oc_steps);
  }
  double t4 = or_now();
  L->t_filter += t1 - t0;
  L->t_solve += t2 - t1;
  L->t_sens += t3 - t2;
  L->t_update += t4 - t3;
  return OR_OK;
}

/* which: 0 x, 1 xfil, 2 xthr, 3 dfds, 4 dgds, 5 val (numeq), 6 node_val */
void or_loop_get(const or_loop *L, int which, double *out)
{
  long n = L->P->nelx;
  switch(which)
  {
  case 0: memcpy(out, L->x, sizeof(double) * n); break;
  case 1: memcpy(out, L->xfil, sizeof(double) * n); break;
  case 2: memcpy(out, L->xthr, sizeof(double) * n); break;
  case 3: memcpy(out, L->dfds, sizeof(double) * n); break;
  case 4: memcpy(out, L->dgds, sizeof(double) * n); break;
  case 5: memcpy(out, L->val, sizeof(double) * L->P->numeq); break;
  case 6: memcpy(out, L->node_val, sizeof(double) * 3 * L->P->numnp); break;
  default: break;
  }
}

/* scalars: compliance, constraint, V0, cg_relres, t_filter, t_solve, t_sens,
   t_update; ints: optstep, cg_iters, oc_steps, mma_outloops */
void or_loop_scalars(const or_loop *L, double *d, int *iv)
{
  d[0] = L->compliance;
  d[1] = L->constraint;
  d[2] = L->V0;
  d[3] = L->cg_relres;
  d[4] = L->t_filter;
  d[5] = L->t_solve;
  d[6] = L->t_sens;
  d[7] = L->t_update;
  d[8] = L->t_pcg;
  iv[0] = L->optstep;
  iv[1] = L->cg_iters;
  iv[2] = L->oc_steps;
  iv[3] = L->mma_outloops;
}

/* ------------------------------------------------------------------------ */
/* 9. Helmholtz PDE filter (FilterHelmholtz, src/optimization/filter_helm.hpp)*/
/*    makeKeFint (:179-223): per element and Gauss point                      */
/*      Ke += (N N^T + B^T (R / (2 sqrt 3))^2 I B) jac,  fe += s N jac,       */
/*    fe /= ipmax for the sensitivity call; densityFilter (:76-138):          */
/*    assemble the nodal scalar system, solve K val = F (Jacobi-PCG here, as  */
/*    "Eigen_CG"), divideToElement (:225-257): sum_gp N . val_e, divided by    */
/*    ipmax for the density call.                                             */
/* ------------------------------------------------------------------------ */
static void or_helm_element(const double *X, double R, double Ke[64], double Nj[8],
                            double Ns[8])
{
  const double g = 1.0 / sqrt(3.0);
  const double c = pow(R / (2 * sqrt(3.0)), 2);
  for(int i = 0; i < 64; i++)
    Ke[i] = 0.0;
  for(int n = 0; n < 8; n++)
    Nj[n] = Ns[n] = 0.0;
  for(int ip = 0; ip < 8; ip++)
  {
    double r[3] = {or_gauss_sign[ip][0] * g, or_gauss_sign[ip][1] * g,
                   or_gauss_sign[ip][2] * g};
    double N[8];
    for(int n = 0; n < 8; n++)
      N[n] = 0.125 * (1.0 + or_gauss_sign[n][0] * r[0]) * (1.0 + or_gauss_sign[n][1] * r[1]) *
             (1.0 + or_gauss_sign[n][2] * r[2]);
    double dN[3][8];
    or_dNdr(r, dN);
    double J[3][3];
    for(int a = 0; a < 3; a++)
      for(int b = 0; b < 3; b++)
      {
        double s = 0.0;
        for(int n = 0; n < 8; n++)
          s += dN[a][n] * X[3 * n + b];
        J[a][b] = s;
      }
    double det = J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) -
                 J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +
                 J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
    double inv[3][3];
    inv[0][0] = (J[1][1] * J[2][2] - J[1][2] * J[2][1]) / det;
    inv[0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) / det;
    inv[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) / det;
    inv[1][0] = (J[1][2] * J[2][0] - J[1][0] * J[2][2]) / det;
    inv[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) / det;
    inv[1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) / det;
    inv[2][0] = (J[1][0] * J[2][1] - J[1][1] * J[2][0]) / det;
    inv[2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) / det;
    inv[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) / det;
    double B[3][8];
    for(int a = 0; a < 3; a++)
      for(int n = 0; n < 8; n++)
      {
        double s = 0.0;
        for(int b = 0; b < 3; b++)
          s += inv[a][b] * dN[b][n];
        B[a][n] = s;
      }
    const double jac = det * 1.0;
    for(int a = 0; a < 8; a++)
      for(int b = 0; b < 8; b++)
      {
        double s = 0.0;
        for(int d = 0; d < 3; d++)
          s += B[d][a] * c * B[d][b];
        Ke[8 * a + b] += (N[a] * N[b] + s) * jac;
      }
    for(int n = 0; n < 8; n++)
    {
      Nj[n] += N[n] * jac;
      Ns[n] += N[n];
    }
  }
}

/* out[nelx] = Helmholtz filter of in[nelx] on the nx x ny x nz box of size
   lx x ly x lz, radius R; sens != 0: the sensitivity call.  Jacobi-PCG from
   zero to ||r|| < tol ||F||. */
int or_helmholtz_filter(int nx, int ny, int nz, double lx, double ly, double lz, double R,
                        const double *in, double *out, int sens, double tol, int maxit,
                        int *iters_out)
{
  if(nx < 1 || ny < 1 || nz < 1 || R <= 0.0)
    return OR_ERR_ARG;
  const long NX = nx + 1, NY = ny + 1, NZ = nz + 1, numnp = NX * NY * NZ;
  const long nelx = (long)nx * ny * nz;
  double *xyz = (double *)malloc(sizeof(double) * 3 * numnp);
  int *conn = (int *)malloc(sizeof(int) * 8 * nelx);
  or_mesh_box(nx, ny, nz, lx, ly, lz, xyz, conn);
  double *K = (double *)calloc(27 * numnp, sizeof(double)); /* [node][neighbour slot] */
  double *F = (double *)calloc(numnp, sizeof(double));
  double Ke[64], Nj[8], Ns[8];
  for(long e = 0; e < nelx; e++)
  {
    double X[24];
    for(int a = 0; a < 8; a++)
      for(int d = 0; d < 3; d++)
        X[3 * a + d] = xyz[3 * (long)conn[8 * e + a] + d];
    or_helm_element(X, R, Ke, Nj, Ns);
    for(int a = 0; a < 8; a++)
    {
      const long na = conn[8 * e + a];
      const long ia = na % NX, ja = (na / NX) % NY, ka = na / (NX * NY);
      for(int b = 0; b < 8; b++)
      {
        const long nb = conn[8 * e + b];
        const long ib = nb % NX, jb = (nb / NX) % NY, kb = nb / (NX * NY);
        const int slot = (int)((kb - ka + 1) * 9 + (jb - ja + 1) * 3 + (ib - ia + 1));
        K[27 * na + slot] += Ke[8 * a + b];
      }
      double fe = in[e] * Nj[a];
      if(sens)
        fe = fe / 8.0;
      F[na] += fe;
    }
  }
  /* Jacobi-PCG */
  double *val = (double *)calloc(numnp, sizeof(double));
  double *r = (double *)malloc(sizeof(double) * numnp);
  double *z = (double *)malloc(sizeof(double) * numnp);
  double *p = (double *)malloc(sizeof(double) * numnp);
  double *Ap = (double *)malloc(sizeof(double) * numnp);
  for(long n = 0; n < numnp; n++)
  {
    r[n] = F[n];
    z[n] = r[n] / K[27 * n + 13];
    p[n] = z[n];
  }
  double bnorm = sqrt(or_dot(F, F, numnp)), zr = or_dot(z, r, numnp);
  int iter = 0;
  while(bnorm > 0.0)
  {
    iter++;
    for(long n = 0; n < numnp; n++)
    {
      const long i = n % NX, j = (n / NX) % NY, k = n / (NX * NY);
      double s = 0.0;
      for(int slot = 0; slot < 27; slot++)
      {
        const double kv = K[27 * n + slot];
        if(kv == 0.0)
          continue;
        const long m = (i + slot % 3 - 1) + (j + (slot / 3) % 3 - 1) * NX +
                       (k + slot / 9 - 1) * NX * NY;
        s += kv * p[m];
      }
      Ap[n] = s;
    }
    const double alpha = zr / or_dot(p, Ap, numnp);
    for(long n = 0; n < numnp; n++)
    {
      val[n] += alpha * p[n];
      r[n] -= alpha * Ap[n];
      z[n] = r[n] / K[27 * n + 13];
    }
    const double zr1 = or_dot(z, r, numnp);
    const double beta = zr1 / zr;
    for(long n = 0; n < numnp; n++)
      p[n] = beta * p[n] + z[n];
    zr = zr1;
    if(sqrt(or_dot(r, r, numnp)) < tol * bnorm || iter > maxit)
      break;
  }
  for(long e = 0; e < nelx; e++)
  {
    double X[24];
    for(int a = 0; a < 8; a++)
      for(int d = 0; d < 3; d++)
        X[3 * a + d] = xyz[3 * (long)conn[8 * e + a] + d];
    or_helm_element(X, R, Ke, Nj, Ns);
    double s = 0.0;
    for(int a = 0; a < 8; a++)
      s += Ns[a] * val[conn[8 * e + a]];
    out[e] = sens ? s : s / 8.0;
  }
  if(iters_out)
    *iters_out = iter;
  free(xyz);
  free(conn);
  free(K);
  free(F);
  free(val);
  free(r);
  free(z);
  free(p);
  free(Ap);
  return OR_OK;
}
