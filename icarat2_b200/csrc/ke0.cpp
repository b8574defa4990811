// Host-side element matrix of the uniform voxel mesh.
//
// Every element of a MeshIcarat box is a translate of element 0, so one
// 24x24 matrix at E = 1 serves the whole grid; the device scales it by
// E(rho_e).  The integration follows LinearElastic::makeKeFint
// (src/problem/elasticity.cpp:211-255): 2x2x2 Gauss rule with points
// +-1/sqrt(3) in Gauss8Cubic order (src/basis/gauss_integration.cpp:268-289),
// trilinear shape-function derivatives (src/basis/shape_function.cpp:422-447),
// B in Voigt order xx,yy,zz,xy,yz,zx (src/basis/bmatrix.hpp:125-140),
// isotropic D from Lame constants (src/problem/elasticity.cpp:72-93),
// Ke = sum B^T D B det(J) w.  Element DOF index = 3 * local node + component.
#include <cmath>
#include <cstring>

namespace icarat_b200
{

// local node coordinates in the reference order 0:(0,0,0) 1:(1,0,0)
// 2:(1,1,0) 3:(0,1,0) 4..7 at z + 1, and the Gauss8Cubic point signs
static const int lc[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0},
                             {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};
static const int gs[8][3] = {{-1, -1, -1}, {1, -1, -1}, {1, 1, -1},
                             {-1, 1, -1},  {-1, -1, 1}, {1, -1, 1},
                             {1, 1, 1},    {-1, 1, 1}};

// isotropic D at E = 1 (Lame constants)
static void elastic_D(double nu, double D[6][6])
{
  const double lam = nu / ((1.0 + nu) * (1.0 - 2.0 * nu));
  const double mu = 1.0 / (2.0 * (1.0 + nu));
  for(int i = 0; i < 6; i++)
    for(int j = 0; j < 6; j++)
      D[i][j] = 0.0;
  for(int i = 0; i < 3; i++)
    for(int j = 0; j < 3; j++)
      D[i][j] = (i == j) ? lam + 2.0 * mu : lam;
  D[3][3] = D[4][4] = D[5][5] = mu;
}

// Voigt B at Gauss point q of the hx x hy x hz voxel; returns det J
static double hexa8_B(double hx, double hy, double hz, int q, double B[6][24])
{
  double X[8][3];
  for(int a = 0; a < 8; a++)
  {
    X[a][0] = lc[a][0] * hx;
    X[a][1] = lc[a][1] * hy;
    X[a][2] = lc[a][2] * hz;
  }
  const double g = 1.0 / std::sqrt(3.0);
  double r[3] = {gs[q][0] * g, gs[q][1] * g, gs[q][2] * g};
  // dN_a/dr_d = 1/8 * s_d(a) * prod_{e != d} (1 + s_e(a) r_e), s = +-1
  double dN[3][8];
  for(int a = 0; a < 8; a++)
  {
    double s[3] = {lc[a][0] ? 1.0 : -1.0, lc[a][1] ? 1.0 : -1.0,
                   lc[a][2] ? 1.0 : -1.0};
    dN[0][a] = 0.125 * s[0] * (1.0 + s[1] * r[1]) * (1.0 + s[2] * r[2]);
    dN[1][a] = 0.125 * s[1] * (1.0 + s[2] * r[2]) * (1.0 + s[0] * r[0]);
    dN[2][a] = 0.125 * s[2] * (1.0 + s[0] * r[0]) * (1.0 + s[1] * r[1]);
  }
  double J[3][3];
  for(int a = 0; a < 3; a++)
    for(int b = 0; b < 3; b++)
    {
      double t = 0.0;
      for(int n = 0; n < 8; n++)
        t += dN[a][n] * X[n][b];
      J[a][b] = t;
    }
  double det = J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) -
               J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +
               J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
  double Ji[3][3];
  Ji[0][0] = (J[1][1] * J[2][2] - J[1][2] * J[2][1]) / det;
  Ji[0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) / det;
  Ji[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) / det;
  Ji[1][0] = (J[1][2] * J[2][0] - J[1][0] * J[2][2]) / det;
  Ji[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) / det;
  Ji[1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) / det;
  Ji[2][0] = (J[1][0] * J[2][1] - J[1][1] * J[2][0]) / det;
  Ji[2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) / det;
  Ji[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) / det;
  double G[3][8];
  for(int a = 0; a < 3; a++)
    for(int n = 0; n < 8; n++)
      G[a][n] = Ji[a][0] * dN[0][n] + Ji[a][1] * dN[1][n] + Ji[a][2] * dN[2][n];
  for(int i = 0; i < 6; i++)
    for(int j = 0; j < 24; j++)
      B[i][j] = 0.0;
  for(int n = 0; n < 8; n++)
  {
    B[0][3 * n] = G[0][n];
    B[1][3 * n + 1] = G[1][n];
    B[2][3 * n + 2] = G[2][n];
    B[3][3 * n] = G[1][n];
    B[3][3 * n + 1] = G[0][n];
    B[4][3 * n + 1] = G[2][n];
    B[4][3 * n + 2] = G[1][n];
    B[5][3 * n] = G[2][n];
    B[5][3 * n + 2] = G[0][n];
  }
  return det;
}

void hexa8_stiffness(double hx, double hy, double hz, double nu, double *ke,
                     double *volume)
{
  double D[6][6];
  elastic_D(nu, D);
  std::memset(ke, 0, sizeof(double) * 576);
  double vol = 0.0;
  for(int q = 0; q < 8; q++)
  {
    double B[6][24];
    const double det = hexa8_B(hx, hy, hz, q, B);
    double BtD[24][6];
    for(int i = 0; i < 24; i++)
      for(int k = 0; k < 6; k++)
      {
        double t = 0.0;
        for(int l = 0; l < 6; l++)
          t += B[l][i] * D[l][k];
        BtD[i][k] = t;
      }
    const double jac = det * 1.0;
    for(int i = 0; i < 24; i++)
      for(int j = 0; j < 24; j++)
      {
        double t = 0.0;
        for(int k = 0; k < 6; k++)
          t += BtD[i][k] * B[k][j];
        ke[24 * i + j] += t * jac;
      }
    vol += jac;
  }
  *volume = vol;
}

// Gauss-averaged stress operator at E = 1: sigma = E(rho) * S u_e with
// S = sum_ip D B(ip) / ipmax (Elastic::makeMisesStress,
// src/problem/elasticity.cpp:166-207, stress_ += De B disp fac); s is 6 x 24
void hexa8_stress_operator(double hx, double hy, double hz, double nu, double *s)
{
  double D[6][6];
  elastic_D(nu, D);
  for(int i = 0; i < 144; i++)
    s[i] = 0.0;
  for(int q = 0; q < 8; q++)
  {
    double B[6][24];
    hexa8_B(hx, hy, hz, q, B);
    for(int i = 0; i < 6; i++)
      for(int j = 0; j < 24; j++)
      {
        double t = 0.0;
        for(int k = 0; k < 6; k++)
          t += D[i][k] * B[k][j];
        s[24 * i + j] += t * (1.0 / 8.0);
      }
  }
}

// Largest eigenvalue of diag(Ke)^-1/2 Ke diag(Ke)^-1/2 by cyclic Jacobi
// rotations.  Since x^T K x = sum_e E_e x_e^T Ke0 x_e <= lmax sum_e E_e
// x_e^T diag(Ke0) x_e = lmax x^T diag(K) x, this bounds lambda_max(D^-1 K)
// of every SIMP stiffness assembled from Ke0 (Dirichlet rows removed or not).
double jacobi_bound(const double *ke)
{
  double A[24][24];
  for(int i = 0; i < 24; i++)
    for(int j = 0; j < 24; j++)
      A[i][j] = ke[24 * i + j] / std::sqrt(ke[24 * i + i] * ke[24 * j + j]);
  for(int sweep = 0; sweep < 60; sweep++)
  {
    double off = 0.0;
    for(int i = 0; i < 24; i++)
      for(int j = i + 1; j < 24; j++)
        off += A[i][j] * A[i][j];
    if(off < 1e-30)
      break;
    for(int p = 0; p < 24; p++)
      for(int q = p + 1; q < 24; q++)
      {
        if(std::fabs(A[p][q]) < 1e-300)
          continue;
        double theta = (A[q][q] - A[p][p]) / (2.0 * A[p][q]);
        double t = (theta >= 0 ? 1.0 : -1.0) /
                   (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
        double cs = 1.0 / std::sqrt(t * t + 1.0), sn = t * cs;
        for(int k = 0; k < 24; k++)
        {
          double akp = A[k][p], akq = A[k][q];
          A[k][p] = cs * akp - sn * akq;
          A[k][q] = sn * akp + cs * akq;
        }
        for(int k = 0; k < 24; k++)
        {
          double apk = A[p][k], aqk = A[q][k];
          A[p][k] = cs * apk - sn * aqk;
          A[q][k] = sn * apk + cs * aqk;
        }
      }
  }
  double lmax = 0.0;
  for(int i = 0; i < 24; i++)
    lmax = A[i][i] > lmax ? A[i][i] : lmax;
  return lmax;
}

} // namespace icarat_b200
