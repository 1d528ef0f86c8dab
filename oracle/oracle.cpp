// CPU oracle for the MSolve Hexa8 solve path -- TEST INFRASTRUCTURE ONLY.
//
// Restates the reference algorithms in FP64 C++ (see oracle.h for the scope
// and the parity status). Compiled with -ffp-contract=off so every product and
// sum is rounded separately, as the reference's C#/.NET and Fortran (no FMA
// contraction) evaluate them. Only tests, the smoke check and the CPU-baseline
// legs of bench.py load this library.
#include "oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// Gauss-Legendre 2-point rule, the reference's 13-digit literals:
// rElHexa8.f90:435-445 and GaussQuadrature.cs:73-81. GP loop order is xi
// outermost, zeta innermost (rElHexa8.f90:449-463, Hexa8.cs:341-363).
const double kGP[2] = {-.5773502691896, .5773502691896};
const double kGW[2] = {1.0, 1.0};
const double kDetTol = 0.00000001;  // rElHexa8.f90:203, Hexa8.cs:16

// CalcH8NablaShape, rElHexa8.f90:25-69 (faDS(1..8)=dN/dxi, (9..16)=dN/deta, (17..24)=dN/dzeta).
void nabla_shape_fortran(double xi, double eta, double zeta, double* ds) {
  const double s = 0.35355339059327376220042218105242;
  double xp = (1.0 + xi) * s, ep = (1.0 + eta) * s, zp = (1.0 + zeta) * s;
  double xm = (1.0 - xi) * s, em = (1.0 - eta) * s, zm = (1.0 - zeta) * s;
  ds[0] = -(em * zm); ds[1] = -ds[0]; ds[2] = ep * zm; ds[3] = -ds[2];
  ds[4] = -(em * zp); ds[5] = -ds[4]; ds[6] = ep * zp; ds[7] = -ds[6];
  ds[8] = -(xm * zm); ds[9] = -(xp * zm); ds[10] = -ds[9]; ds[11] = -ds[8];
  ds[12] = -(xm * zp); ds[13] = -(xp * zp); ds[14] = -ds[13]; ds[15] = -ds[12];
  ds[16] = -(xm * em); ds[17] = -(xp * em); ds[18] = -(xp * ep); ds[19] = -(xm * ep);
  ds[20] = -ds[16]; ds[21] = -ds[17]; ds[22] = -ds[18]; ds[23] = -ds[19];
}

// CalcH8Shape, rElHexa8.f90:93-117 (and Hexa8.cs:137-157, same constants).
void shape(double xi, double eta, double zeta, double* s8) {
  const double c = 0.5;
  double xp = (1.0 + xi) * c, ep = (1.0 + eta) * c, zp = (1.0 + zeta) * c;
  double xm = (1.0 - xi) * c, em = (1.0 - eta) * c, zm = (1.0 - zeta) * c;
  s8[0] = xm * em * zm; s8[1] = xp * em * zm; s8[2] = xp * ep * zm; s8[3] = xm * ep * zm;
  s8[4] = xm * em * zp; s8[5] = xp * em * zp; s8[6] = xp * ep * zp; s8[7] = xm * ep * zp;
}

// CalcH8JDetJ, rElHexa8.f90:141-208: J[a][i] = sum_n dN_a,n * x_n,i (a natural, i physical).
int jdetj_fortran(const double* xyz, const double* ds, double* J, double* det) {
  for (int a = 0; a < 3; ++a)
    for (int i = 0; i < 3; ++i) {
      double s = ds[8 * a + 0] * xyz[0 * 3 + i];
      for (int n = 1; n < 8; ++n) s = s + ds[8 * a + n] * xyz[n * 3 + i];
      J[3 * a + i] = s;
    }
  double d1 = J[0] * (J[4] * J[8] - J[7] * J[5]);
  double d2 = -J[1] * (J[3] * J[8] - J[6] * J[5]);
  double d3 = J[2] * (J[3] * J[7] - J[6] * J[4]);
  *det = d1 + d2 + d3;
  return (*det < kDetTol) ? -1001 : 0;  // iErrNegDet, hCommon.h:29
}

// CalcH8B, rElHexa8.f90:232-397. B rows: exx, eyy, ezz, gxy, gyz, gzx; columns node-major x,y,z.
void b_matrix_fortran(double det, const double* J, const double* ds, double* B /*[6][24]*/) {
  double inv = 1.0 / det;
  // faJInv(r,c) with r,c 1-based -> Ji[3*(r-1)+(c-1)]; J(a,i) -> J[3*(a-1)+(i-1)]
  double Ji[9];
  Ji[0] = (J[4] * J[8] - J[7] * J[5]) * inv;  // (1,1)
  Ji[3] = (J[6] * J[5] - J[3] * J[8]) * inv;  // (2,1)
  Ji[6] = (J[3] * J[7] - J[6] * J[4]) * inv;  // (3,1)
  Ji[1] = (J[7] * J[2] - J[1] * J[8]) * inv;  // (1,2)
  Ji[4] = (J[0] * J[8] - J[6] * J[2]) * inv;  // (2,2)
  Ji[7] = (J[6] * J[1] - J[7] * J[0]) * inv;  // (3,2)
  Ji[2] = (J[1] * J[5] - J[4] * J[2]) * inv;  // (1,3)
  Ji[5] = (J[3] * J[2] - J[0] * J[5]) * inv;  // (2,3)
  Ji[8] = (J[0] * J[4] - J[3] * J[1]) * inv;  // (3,3)
  std::memset(B, 0, sizeof(double) * 144);
  for (int n = 0; n < 8; ++n) {
    double bx = Ji[0] * ds[n] + Ji[1] * ds[8 + n] + Ji[2] * ds[16 + n];
    double by = Ji[3] * ds[n] + Ji[4] * ds[8 + n] + Ji[5] * ds[16 + n];
    double bz = Ji[6] * ds[n] + Ji[7] * ds[8 + n] + Ji[8] * ds[16 + n];
    B[0 * 24 + 3 * n + 0] = bx;
    B[1 * 24 + 3 * n + 1] = by;
    B[2 * 24 + 3 * n + 2] = bz;
    B[3 * 24 + 3 * n + 0] = by; B[3 * 24 + 3 * n + 1] = bx;
    B[4 * 24 + 3 * n + 1] = bz; B[4 * 24 + 3 * n + 2] = by;
    B[5 * 24 + 3 * n + 0] = bz; B[5 * 24 + 3 * n + 2] = bx;
  }
}

// K += w * B^T D B over one Gauss point, packed row-wise upper (I <= J),
// CalcH8K rElHexa8.f90:489-543 and Hexa8.StiffnessMatrix Hexa8.cs:368-401.
void add_btdb(const double* D, const double* B, double w, double* K300) {
  int ks = 0;
  for (int i = 0; i < 24; ++i) {
    double eb[6];
    for (int k = 0; k < 6; ++k) {
      double s = D[6 * k + 0] * B[0 * 24 + i];
      for (int l = 1; l < 6; ++l) s = s + D[6 * k + l] * B[l * 24 + i];
      eb[k] = s;
    }
    for (int j = i; j < 24; ++j) {
      double s = B[0 * 24 + j] * eb[0];
      for (int k = 1; k < 6; ++k) s = s + B[k * 24 + j] * eb[k];
      K300[ks] = K300[ks] + s * w;
      ++ks;
    }
  }
}

// Hexa8.CalculateShapeDerivativeValues, Hexa8.cs:284-330 ("Alex code" C# path).
void nabla_shape_csharp(double xi, double eta, double zeta, double* dxi, double* deta, double* dzeta) {
  const double e8 = 0.125;
  double xp = 1.0 + xi, ep = 1.0 + eta, zp = 1.0 + zeta;
  double xm = 1.0 - xi, em = 1.0 - eta, zm = 1.0 - zeta;
  dxi[0] = -e8 * em * zm; dxi[1] = -dxi[0]; dxi[2] = e8 * ep * zm; dxi[3] = -dxi[2];
  dxi[4] = -e8 * em * zp; dxi[5] = -dxi[4]; dxi[6] = e8 * ep * zp; dxi[7] = -dxi[6];
  deta[0] = -e8 * xm * zm; deta[1] = -e8 * xp * zm; deta[2] = -deta[1]; deta[3] = -deta[0];
  deta[4] = -e8 * xm * zp; deta[5] = -e8 * xp * zp; deta[6] = -deta[5]; deta[7] = -deta[4];
  dzeta[0] = -e8 * xm * em; dzeta[1] = -e8 * xp * em; dzeta[2] = -e8 * xp * ep; dzeta[3] = -e8 * xm * ep;
  dzeta[4] = -dzeta[0]; dzeta[5] = -dzeta[1]; dzeta[6] = -dzeta[2]; dzeta[7] = -dzeta[3];
}

int h8_stiffness_fortran_impl(const double* xyz, const double* D8 /*8 x 36*/, double* K300) {
  double w[8], S[64], DS[192], J[72], det[8], B[8 * 144];
  int st = orc_h8_gauss_matrices(xyz, w, S, DS, J, det, B);
  orc_h8_k(D8, B, w, K300);
  return st;
}

}  // namespace

extern "C" {

int orc_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

// ElasticMaterial3D.GetConstitutiveMatrix, ElasticMaterial3D.cs:20-44
// (StochasticElasticMaterial3D.cs:26-53 is the same with a field-valued E).
void orc_elastic_D(double E, double nu, double* D) {
  double e1 = E / (1.0 + nu);
  double e2 = e1 * nu / (1.0 - 2.0 * nu);
  double e3 = e1 + e2;
  double e4 = e1 * 0.5;
  for (int i = 0; i < 36; ++i) D[i] = 0.0;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) D[6 * i + j] = (i == j) ? e3 : e2;
  D[21] = e4; D[28] = e4; D[35] = e4;
}

// CalcH8GaussMatrices, rElHexa8.f90:422-464. Layouts (C order): S[8][8],
// DS[8][24], J[8][3][3] (J[m][a][i]), detJ[8], B[8][6][24]. Returns 0 or
// -1001 if any Gauss point has detJ < 1e-8 (the Fortran prints and goes on).
int orc_h8_gauss_matrices(const double* xyz, double* w, double* S, double* DS, double* J,
                          double* det, double* B) {
  int st = 0, m = 0;
  for (int ix = 0; ix < 2; ++ix)
    for (int iy = 0; iy < 2; ++iy)
      for (int iz = 0; iz < 2; ++iz, ++m) {
        double xi = kGP[ix], eta = kGP[iy], zeta = kGP[iz];
        nabla_shape_fortran(xi, eta, zeta, DS + 24 * m);
        shape(xi, eta, zeta, S + 8 * m);
        int e = jdetj_fortran(xyz, DS + 24 * m, J + 9 * m, det + m);
        if (e) st = e;
        b_matrix_fortran(det[m], J + 9 * m, DS + 24 * m, B + 144 * m);
        w[m] = kGW[ix] * kGW[iy] * kGW[iz] * det[m];
      }
  return st;
}

// CalcH8K, rElHexa8.f90:489-543; Emat[8][6][6], B[8][6][24], weight[8].
void orc_h8_k(const double* Emat, const double* B, const double* w, double* K300) {
  for (int i = 0; i < 300; ++i) K300[i] = 0.0;
  for (int m = 0; m < 8; ++m) add_btdb(Emat + 36 * m, B + 144 * m, w[m], K300);
}

// Hexa8WithStochasticMaterial.StiffnessMatrix (Hexa8WithStochasticMaterial.cs:61-110):
// D at every Gauss point from the element's E, then CalcH8GaussMatrices + CalcH8K.
int orc_h8_stiffness_fortran(const double* xyz, double E, double nu, double* K300) {
  double D8[8 * 36];
  orc_elastic_D(E, nu, D8);
  for (int m = 1; m < 8; ++m) std::memcpy(D8 + 36 * m, D8, sizeof(double) * 36);
  return h8_stiffness_fortran_impl(xyz, D8, K300);
}

// Hexa8.StiffnessMatrix "Alex code" path, Hexa8.cs:256-401 with Jacobian3D.cs:23-118.
int orc_h8_stiffness_csharp(const double* xyz, double E, double nu, double* K300) {
  double D[36];
  orc_elastic_D(E, nu, D);
  for (int i = 0; i < 300; ++i) K300[i] = 0.0;
  int st = 0;
  for (int ix = 0; ix < 2; ++ix)
    for (int iy = 0; iy < 2; ++iy)
      for (int iz = 0; iz < 2; ++iz) {
        double dxi[8], deta[8], dzeta[8];
        nabla_shape_csharp(kGP[ix], kGP[iy], kGP[iz], dxi, deta, dzeta);
        // Jacobian3D.CalculateJacobianMatrix, :93-107 (accumulates from 0 over nodes)
        double m[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        for (int n = 0; n < 8; ++n)
          for (int j = 0; j < 3; ++j) {
            m[0 + j] = m[0 + j] + xyz[3 * n + j] * dxi[n];
            m[3 + j] = m[3 + j] + xyz[3 * n + j] * deta[n];
            m[6 + j] = m[6 + j] + xyz[3 * n + j] * dzeta[n];
          }
        // CalculateJacobianDeterminant, :109-118
        double d1 = m[0] * ((m[4] * m[8]) - (m[7] * m[5]));
        double d2 = m[1] * ((m[3] * m[8]) - (m[6] * m[5]));
        double d3 = m[2] * ((m[3] * m[7]) - (m[6] * m[4]));
        double det = d1 - d2 + d3;
        if (det < 0) st = -1001;
        // CalculateJacobianInverse, :51-74
        double di = 1.0 / det, ji[9];
        ji[0] = ((m[4] * m[8]) - (m[7] * m[5])) * di;
        ji[1] = ((m[7] * m[2]) - (m[1] * m[8])) * di;
        ji[2] = ((m[1] * m[5]) - (m[4] * m[2])) * di;
        ji[3] = ((m[6] * m[5]) - (m[3] * m[8])) * di;
        ji[4] = ((m[0] * m[8]) - (m[6] * m[2])) * di;
        ji[5] = ((m[3] * m[2]) - (m[0] * m[5])) * di;
        ji[6] = ((m[3] * m[7]) - (m[6] * m[4])) * di;
        ji[7] = ((m[6] * m[1]) - (m[7] * m[0])) * di;
        ji[8] = ((m[0] * m[4]) - (m[3] * m[1])) * di;
        // CalculateDeformationMatrix, Hexa8.cs:256-282
        double B[144];
        std::memset(B, 0, sizeof(B));
        for (int s = 0; s < 8; ++s) {
          double bx = (ji[0] * dxi[s]) + (ji[1] * deta[s]) + (ji[2] * dzeta[s]);
          double by = (ji[3] * dxi[s]) + (ji[4] * deta[s]) + (ji[5] * dzeta[s]);
          double bz = (ji[6] * dxi[s]) + (ji[7] * deta[s]) + (ji[8] * dzeta[s]);
          B[0 * 24 + 3 * s] = bx; B[1 * 24 + 3 * s + 1] = by; B[2 * 24 + 3 * s + 2] = bz;
          B[3 * 24 + 3 * s] = by; B[3 * 24 + 3 * s + 1] = bx;
          B[4 * 24 + 3 * s + 1] = bz; B[4 * 24 + 3 * s + 2] = by;
          B[5 * 24 + 3 * s] = bz; B[5 * 24 + 3 * s + 2] = bx;
        }
        double wf = kGW[ix] * kGW[iy] * kGW[iz] * det;
        add_btdb(D, B, wf, K300);
      }
  return st;
}

// Hexa8.CalculateConsistentMass, Hexa8.cs:403-435 (packed row-wise upper, 300).
int orc_h8_consistent_mass(const double* xyz, double rho, double* M300) {
  double w[8], S[64], DS[192], J[72], det[8], B[8 * 144];
  int st = orc_h8_gauss_matrices(xyz, w, S, DS, J, det, B);
  double M[24][24];
  std::memset(M, 0, sizeof(M));
  for (int g = 0; g < 8; ++g) {
    double wd = w[g] * rho;
    const double* N = S + 8 * g;
    for (int I = 0; I < 8; ++I)
      for (int Jn = I; Jn < 8; ++Jn) M[3 * I][3 * Jn] = M[3 * I][3 * Jn] + N[I] * N[Jn] * wd;
  }
  for (int I = 0; I < 8; ++I)
    for (int Jn = I; Jn < 8; ++Jn) {
      M[3 * I + 1][3 * Jn + 1] = M[3 * I][3 * Jn];
      M[3 * I + 2][3 * Jn + 2] = M[3 * I][3 * Jn];
    }
  int ks = 0;
  for (int i = 0; i < 24; ++i)
    for (int j = i; j < 24; ++j) M300[ks++] = M[i][j];
  return st;
}

// CalcH8Strains (rElHexa8.f90:636-648): strains[m] = MatMul(B_m, u), each row
// summed over the 24 columns in order.
void orc_h8_strains(const double* B /*[8][6][24]*/, const double* u24, double* strains /*[8][6]*/) {
  for (int m = 0; m < 8; ++m)
    for (int row = 0; row < 6; ++row) {
      double s = 0.0;
      for (int col = 0; col < 24; ++col) s = s + B[144 * m + 24 * row + col] * u24[col];
      strains[6 * m + row] = s;
    }
}

// Hexa8.CalculateStresses + CalculateForces (Hexa8.cs:453-510) with
// ElasticMaterial3D (ElasticMaterial3D.cs:20-44, 75-81: UpdateMaterial stores
// the strain increment, stresses = D * increment, Matrix2D * Vector row by row)
// and CalcH8Forces (rElHexa8.f90:724-747: forces += w_m * B_m^T stresses_m,
// Gauss points xi outer, zeta inner). du == NULL: du = u. Outputs may be NULL.
int orc_h8_stress(const double* xyz, double E, double nu, const double* u, const double* du, double* strains48,
                  double* stresses48, double* forces24) {
  double w[8], S[64], DS[192], J[72], det[8], B[8 * 144];
  int st = orc_h8_gauss_matrices(xyz, w, S, DS, J, det, B);
  double eps[48], deps[48], sig[48], D[36];
  orc_h8_strains(B, u, eps);
  orc_h8_strains(B, du ? du : u, deps);
  orc_elastic_D(E, nu, D);
  for (int m = 0; m < 8; ++m)
    for (int row = 0; row < 6; ++row) {
      double s = 0.0;
      for (int col = 0; col < 6; ++col) s = s + D[6 * row + col] * deps[6 * m + col];
      sig[6 * m + row] = s;
    }
  if (strains48) std::memcpy(strains48, eps, sizeof(eps));
  if (stresses48) std::memcpy(stresses48, sig, sizeof(sig));
  if (forces24) {
    for (int i = 0; i < 24; ++i) forces24[i] = 0.0;
    for (int m = 0; m < 8; ++m)
      for (int i = 0; i < 24; ++i) {
        double s = 0.0;
        for (int row = 0; row < 6; ++row) s = s + B[144 * m + 24 * row + i] * sig[6 * m + row];
        forces24[i] = forces24[i] + w[m] * s;
      }
  }
  return st;
}

void orc_h8_stress_batch(int n, const double* xyz, const double* E, double nu, const double* u, const double* du,
                         double* strains, double* stresses, double* forces, int* status) {
  int st = 0;
#pragma omp parallel for schedule(static) reduction(min : st)
  for (int e = 0; e < n; ++e) {
    const int64_t k = e;
    int s = orc_h8_stress(xyz + 24 * k, E[e], nu, u + 24 * k, du ? du + 24 * k : nullptr,
                          strains ? strains + 48 * k : nullptr, stresses ? stresses + 48 * k : nullptr,
                          forces ? forces + 24 * k : nullptr);
    if (s < st) st = s;
  }
  if (status) *status = st;
}

void orc_h8_stiffness_batch(int n, const double* xyz, const double* E, double nu, double* K, int* status) {
  int st = 0;
#pragma omp parallel for schedule(static) reduction(min : st)
  for (int e = 0; e < n; ++e) {
    int s = orc_h8_stiffness_fortran(xyz + 24 * (int64_t)e, E[e], nu, K + 300 * (int64_t)e);
    if (s < st) st = s;
  }
  if (status) *status = st;
}

// Hexa8MeshGenerator.BuildNodes (:508-568): IDs x fastest, then y, then z.
void orc_block_nodes(int nx, int ny, int nz, double h, double* xyz) {
  int64_t id = 0;
  for (int k = 0; k <= nz; ++k)
    for (int j = 0; j <= ny; ++j)
      for (int i = 0; i <= nx; ++i, ++id) {
        xyz[3 * id + 0] = i * h; xyz[3 * id + 1] = j * h; xyz[3 * id + 2] = k * h;
      }
}

// Element connectivity, Hexa8MeshGenerator.cs:1075-1089 (0-based node indices):
// bottom face (z) counter-clockwise n1..n4 from the element origin, then the top face.
void orc_block_conn(int nx, int ny, int nz, int* conn) {
  int64_t e = 0;
  int X = nx + 1, XY = (nx + 1) * (ny + 1);
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i, ++e) {
        int b = k * XY + j * X + i;
        int* c = conn + 8 * e;
        c[0] = b; c[1] = b + 1; c[2] = b + X + 1; c[3] = b + X;
        c[4] = b + XY; c[5] = b + XY + 1; c[6] = b + XY + X + 1; c[7] = b + XY + X;
      }
}

// Model.EnumerateGlobalDOFs (Model.cs:165-215) / Subdomain.EnumerateDOFs
// (Subdomain.cs:77-135): ascending node ID, X,Y,Z per node, constrained -> -1.
int orc_enumerate_dofs(int n_nodes, const uint8_t* cons, int* dof) {
  int n = 0;
  for (int i = 0; i < n_nodes; ++i)
    for (int c = 0; c < 3; ++c) dof[3 * i + c] = cons[3 * i + c] ? -1 : n++;
  return n;
}

// GlobalMatrixAssemblerSkyline.CalculateRowIndex, :14-42 (rowIndex[1]=1 hard-coded).
int64_t orc_skyline_rowindex(int n_elems, const int* conn, const int* dof3, int n_dofs, int64_t* rowIndex) {
  std::vector<int64_t> h(n_dofs, 0);
  for (int e = 0; e < n_elems; ++e) {
    int mn = INT32_MAX;
    for (int a = 0; a < 8; ++a)
      for (int c = 0; c < 3; ++c) {
        int d = dof3[3 * conn[8 * e + a] + c];
        if (d != -1) mn = std::min(mn, d);
      }
    for (int a = 0; a < 8; ++a)
      for (int c = 0; c < 3; ++c) {
        int d = dof3[3 * conn[8 * e + a] + c];
        if (d != -1) h[d] = std::max<int64_t>(h[d], (int64_t)d - mn);
      }
  }
  rowIndex[0] = 0;
  if (n_dofs >= 1) rowIndex[1] = 1;
  for (int i = 1; i < n_dofs; ++i) rowIndex[i + 1] = rowIndex[i] + h[i] + 1;
  return rowIndex[n_dofs];
}

// GlobalMatrixAssemblerSkyline.CalculateGlobalMatrix scatter, :60-101:
// Data[RowIndex[dofRow] + (dofRow - dofCol)] += K_e[i][j] for dofRow >= dofCol.
void orc_skyline_assemble(int n_elems, const int* conn, const int* dof3, const double* Ke,
                          const int64_t* rowIndex, double* data) {
  for (int e = 0; e < n_elems; ++e) {
    const double* k = Ke + 300 * (int64_t)e;
    int d[24];
    for (int a = 0; a < 8; ++a)
      for (int c = 0; c < 3; ++c) d[3 * a + c] = dof3[3 * conn[8 * e + a] + c];
    for (int i = 0; i < 24; ++i) {
      if (d[i] == -1) continue;
      for (int j = 0; j < 24; ++j) {
        if (d[j] == -1) continue;
        int64_t hgt = (int64_t)d[i] - d[j];
        if (hgt < 0) continue;
        int r = std::min(i, j), c = std::max(i, j);
        int64_t idx = 300 - (int64_t)(24 - r + 1) * (24 - r) / 2 + c - r;  // SymmetricMatrix2D.IndexOf :44-49
        data[rowIndex[d[i]] + hgt] = data[rowIndex[d[i]] + hgt] + k[idx];
      }
    }
  }
}

// SkylineMatrix2D.Factorize, :63-159 (active-column LDL^T, in place; D on the
// diagonal, unit-L multipliers in the envelope). Zero pivots below tol are
// recorded as zero-energy modes (count only) and the pivot set to 1, as the
// reference does. Returns 0, or -1 on a near-zero reduced diagonal (:109).
int orc_skyline_factorize(int n, const int64_t* ri, double* d, double tol, int* n_zems) {
  int kfix = 0;
  for (int nn = 0; nn < n; ++nn) {
    int64_t KN = ri[nn], KL = KN + 1, KU = ri[nn + 1] - 1, KH = KU - KL;
    if (KH < 0) continue;
    int64_t K;
    if (KH > 0) {
      K = nn - KH;
      int64_t KLT = KU;
      for (int64_t j = 0; j < KH; ++j) {
        KLT--;
        int64_t KI = ri[K];
        int64_t ND = ri[K + 1] - KI - 1;
        if (ND > 0) {
          int64_t KK = std::min<int64_t>(j + 1, ND);
          double C = 0;
          for (int64_t l = 1; l <= KK; ++l) C += d[KI + l] * d[KLT + l];
          d[KLT] -= C;
        }
        K++;
      }
    }
    K = nn;
    double B = 0;
    for (int64_t KK = KL; KK <= KU; ++KK) {
      K--;
      int64_t KI = ri[K];
      if (std::fabs(d[KI]) < tol) return -1;
      double C = d[KK] / d[KI];
      B += C * d[KK];
      d[KK] = C;
    }
    d[KN] -= B;
    if (std::fabs(d[KN]) < tol) {
      d[KN] = 1;
      for (int64_t i1 = KN + 1; i1 <= KU; ++i1) d[i1] = 0;
      for (int irest = nn + 1; irest < n; ++irest) {
        int64_t m1 = ri[irest] + irest - nn;
        if (m1 <= ri[irest + 1]) d[m1] = 0;
      }
      kfix++;
    }
  }
  if (n_zems) *n_zems = kfix;
  return 0;
}

// SkylineMatrix2D.Solve, :161-212: forward reduction, diagonal scaling, back substitution.
void orc_skyline_solve(int n, const int64_t* ri, const double* d, const double* f, double* x) {
  for (int i = 0; i < n; ++i) x[i] = f[i];
  for (int nn = 0; nn < n; ++nn) {
    int64_t KL = ri[nn] + 1, KU = ri[nn + 1] - 1;
    if (KU >= KL) {
      int64_t k = nn;
      double C = 0;
      for (int64_t KK = KL; KK <= KU; ++KK) { k--; C += d[KK] * x[k]; }
      x[nn] -= C;
    }
  }
  for (int nn = 0; nn < n; ++nn) x[nn] /= d[ri[nn]];
  int nn = n - 1;
  for (int l = 1; l < n; ++l) {
    int64_t KL = ri[nn] + 1, KU = ri[nn + 1] - 1;
    if (KU >= KL) {
      int64_t k = nn;
      for (int64_t KK = KL; KK <= KU; ++KK) { k--; x[k] -= d[KK] * x[nn]; }
    }
    nn--;
  }
}

// SkylineMatrix2D.Multiply, :224-286 (symmetric envelope product).
void orc_skyline_multiply(int n, const int64_t* ri, const double* d, const double* x, double* y) {
  for (int i = 0; i < n; ++i) y[i] = 0;
  int64_t pos = 0;
  for (int i = 0; i < n; ++i) {
    int64_t height = ri[i + 1] - ri[i];
    if (height <= 0) continue;
    y[i] += d[pos] * x[i];
    pos++;
    for (int64_t j = 0; j < height - 1; ++j) {
      int64_t row = i - j - 1;
      y[row] += d[pos] * x[i];
      y[i] += d[pos] * x[row];
      pos++;
    }
  }
}

// CSR pattern over free DOFs: the columns of DOF row d are all free DOFs of
// the nodes sharing an element with d's node, ascending. Returns nnz.
int64_t orc_csr_pattern(int n_nodes, int n_elems, const int* conn, const int* dof3, int n_dofs,
                        int64_t* rowptr, int* colind) {
  std::vector<std::vector<int>> adj(n_nodes);
  for (int e = 0; e < n_elems; ++e)
    for (int a = 0; a < 8; ++a)
      for (int b = 0; b < 8; ++b) adj[conn[8 * e + a]].push_back(conn[8 * e + b]);
  for (auto& v : adj) {
    std::sort(v.begin(), v.end());
    v.erase(std::unique(v.begin(), v.end()), v.end());
  }
  int64_t nnz = 0;
  rowptr[0] = 0;
  for (int nd = 0; nd < n_nodes; ++nd)
    for (int c = 0; c < 3; ++c) {
      int d = dof3[3 * nd + c];
      if (d < 0) continue;
      for (int m : adj[nd])
        for (int c2 = 0; c2 < 3; ++c2) {
          int d2 = dof3[3 * m + c2];
          if (d2 < 0) continue;
          if (colind) colind[nnz] = d2;
          nnz++;
        }
      rowptr[d + 1] = nnz;
    }
  (void)n_dofs;
  return nnz;
}

void orc_csr_assemble(int n_elems, const int* conn, const int* dof3, const double* Ke,
                      const int64_t* rowptr, const int* colind, double* val) {
  for (int e = 0; e < n_elems; ++e) {
    const double* k = Ke + 300 * (int64_t)e;
    int d[24];
    for (int a = 0; a < 8; ++a)
      for (int c = 0; c < 3; ++c) d[3 * a + c] = dof3[3 * conn[8 * e + a] + c];
    for (int i = 0; i < 24; ++i) {
      if (d[i] < 0) continue;
      const int* b = colind + rowptr[d[i]];
      const int* en = colind + rowptr[d[i] + 1];
      for (int j = 0; j < 24; ++j) {
        if (d[j] < 0) continue;
        int r = std::min(i, j), c = std::max(i, j);
        int idx = 300 - (24 - r + 1) * (24 - r) / 2 + c - r;
        int64_t p = std::lower_bound(b, en, d[j]) - colind;
        val[p] = val[p] + k[idx];
      }
    }
  }
}

void orc_csr_multiply(int n, const int64_t* rp, const int* ci, const double* v, const double* x, double* y) {
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; ++i) {
    double s = 0;
    for (int64_t p = rp[i]; p < rp[i + 1]; ++p) s += v[p] * x[ci[p]];
    y[i] = s;
  }
}

}  // extern "C"

namespace {

double dot(int n, const double* a, const double* b) {
  double s = 0;
#pragma omp parallel for schedule(static) reduction(+ : s)
  for (int i = 0; i < n; ++i) s += a[i] * b[i];
  return s;
}

// SolverPCG.Solve, PCG/SolverPCG.cs:105-149, with the simple search vector of
// SolverPCGSimpleSearchVectorCalculator.cs:18-41 and the zero start of
// SolverPCGMatrixInitialization / SolverPCGSkyline.Initialize (x0 = 0, r0 = b,
// detf = ||b||). `iterations` is the reference's value (the loop index at the
// break, i.e. one less than the number of matrix products when converged).
template <class MatVec, class Precond>
int pcg(int n, MatVec A, Precond M, const double* b, double* x, int max_it, double tol,
        int* iterations, int* matvecs, double* rel_res) {
  std::vector<double> r(b, b + n), z(n, 0.0), p(n, 0.0), q(n, 0.0);
  for (int i = 0; i < n; ++i) x[i] = 0.0;
  double detf = std::sqrt(dot(n, b, b));
  int it = 0, mv = 0;
  double err = 0.0;
  double zr_old = 0.0;
  if (std::sqrt(dot(n, r.data(), r.data())) > 1e-25) {
    M(r.data(), z.data());
    for (it = 0; it < max_it; ++it) {
      double zr = dot(n, z.data(), r.data());
      if (it > 0) {
        double beta = zr / zr_old;
#pragma omp parallel for schedule(static)
        for (int i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
      } else {
        for (int i = 0; i < n; ++i) p[i] = z[i];
      }
      zr_old = zr;
      A(p.data(), q.data());
      ++mv;
      double a = zr / dot(n, p.data(), q.data());
      double detz = 0;
#pragma omp parallel for schedule(static) reduction(+ : detz)
      for (int i = 0; i < n; ++i) {
        r[i] -= a * q[i];
        x[i] += a * p[i];
        detz += r[i] * r[i];
      }
      err = std::sqrt(detz) / detf;
      if (err < tol) break;
      M(r.data(), z.data());
    }
  }
  if (iterations) *iterations = it;
  if (matvecs) *matvecs = mv;
  if (rel_res) *rel_res = err;
  return (mv > 0 && err >= tol) ? -2001 : 0;
}

}  // namespace

extern "C" {

// Jacobi-preconditioned PCG on a CSR matrix. The diagonal preconditioner
// z_j = r_j / K_jj follows PolynomialChaosSolverPCGMatrixCalculator.PreconditionDiagonal
// (:467-495); the loop is SolverPCG.Solve.
// SolverPCG (SolverPCG.cs:105-149) with SolverPCGReorthogonalizationSearchVectorCalculator
// (SearchVectors.cs:13-166): p = z - sum_c (z.q_c / p_c.q_c) p_c over every stored
// pair, gradient (p.r)/(p.q), the pair appended to the store (P, Q [cap][n], pq
// [cap], *count pairs in use). start: InitializeStartingVectorFromReorthogonalized-
// SearchVectors drops the last pair and sets x0 = sum_c (p_c.b / p_c.q_c) p_c,
// then r0 = b - K x0 (start = 2: the store is emptied after x0, for a matrix
// other than the one the pairs came from). Jacobi preconditioner on the CSR diagonal. Returns 0,
// -2001 (not converged) or -1 (store full).
int orc_pcg_reorth_csr(int n, const int64_t* rp, const int* ci, const double* v, const double* b, double* x,
                       double* P, double* Q, double* pq, int cap, int* count, int start, int max_it, double tol,
                       int* iterations, double* rel_res) {
  std::vector<double> dinv(n), r(n), z(n), p(n), q(n);
  for (int i = 0; i < n; ++i) {
    double dd = 0;
    for (int64_t k = rp[i]; k < rp[i + 1]; ++k)
      if (ci[k] == i) dd = v[k];
    dinv[i] = 1.0 / dd;
  }
  int k = *count;
  const double detf = std::sqrt(dot(n, b, b));
  for (int i = 0; i < n; ++i) x[i] = 0.0;
  if (start && k > 0) --k;
  if (start && k > 0) {
    for (int c = 0; c < k; ++c) {
      const double* pc = P + (int64_t)c * n;
      double a = 0, bt = 0;
      for (int i = 0; i < n; ++i) {
        a += pc[i] * Q[(int64_t)c * n + i];
        bt += pc[i] * b[i];
      }
      const double vv = bt / a;
      for (int i = 0; i < n; ++i) x[i] += vv * pc[i];
    }
    orc_csr_multiply(n, rp, ci, v, x, q.data());
    for (int i = 0; i < n; ++i) r[i] = b[i] - q[i];
    if (start == 2) k = 0;  // the pairs belong to another matrix: start a fresh store
  } else {
    for (int i = 0; i < n; ++i) r[i] = b[i];
  }
  int it = 0, st = 0;
  double err = std::sqrt(dot(n, r.data(), r.data())) / detf;
  if (std::sqrt(dot(n, r.data(), r.data())) > 1e-25) {
    for (int i = 0; i < n; ++i) z[i] = r[i] * dinv[i];
    st = -2001;
    for (it = 0; it < max_it; ++it) {
      if (k >= cap) {
        st = -1;
        break;
      }
      for (int i = 0; i < n; ++i) p[i] = z[i];
      for (int c = 0; c < k; ++c) {
        const double* pc = P + (int64_t)c * n;
        const double* qc = Q + (int64_t)c * n;
        double a = 0, bb = 0;
        for (int i = 0; i < n; ++i) {
          a += z[i] * qc[i];
          bb += pc[i] * qc[i];
        }
        const double ab = a / bb;
        for (int i = 0; i < n; ++i) p[i] -= ab * pc[i];
      }
      orc_csr_multiply(n, rp, ci, v, p.data(), q.data());
      const double pr = dot(n, p.data(), r.data()), pqv = dot(n, p.data(), q.data());
      std::memcpy(P + (int64_t)k * n, p.data(), sizeof(double) * n);
      std::memcpy(Q + (int64_t)k * n, q.data(), sizeof(double) * n);
      pq[k] = pqv;
      ++k;
      const double a = pr / pqv;
      double detz = 0;
      for (int i = 0; i < n; ++i) {
        r[i] -= a * q[i];
        x[i] += a * p[i];
        detz += r[i] * r[i];
      }
      err = std::sqrt(detz) / detf;
      if (err < tol) {
        st = 0;
        break;
      }
      for (int i = 0; i < n; ++i) z[i] = r[i] * dinv[i];
    }
  }
  *count = k;
  if (iterations) *iterations = it;
  if (rel_res) *rel_res = err;
  return st;
}

int orc_pcg_csr_jacobi(int n, const int64_t* rp, const int* ci, const double* v, const double* b,
                       double* x, int max_it, double tol, int* iterations, int* matvecs, double* rel_res) {
  std::vector<double> dinv(n);
  for (int i = 0; i < n; ++i) {
    double dd = 0;
    for (int64_t p = rp[i]; p < rp[i + 1]; ++p)
      if (ci[p] == i) dd = v[p];
    dinv[i] = 1.0 / dd;
  }
  auto A = [&](const double* in, double* out) { orc_csr_multiply(n, rp, ci, v, in, out); };
  auto M = [&](const double* in, double* out) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) out[i] = in[i] * dinv[i];
  };
  return pcg(n, A, M, b, x, max_it, tol, iterations, matvecs, rel_res);
}

// PCG on a skyline matrix preconditioned by a factorised skyline
// (MonteCarloSolverPCGDirectMatrixCalculator.cs:38-51: matvec = skyline
// Multiply, preconditioner = LDL^T solve of the cached first-realization K).
int orc_pcg_skyline(int n, const int64_t* ri, const double* data, const double* ldlt, const double* b,
                    double* x, int max_it, double tol, int* iterations, int* matvecs, double* rel_res) {
  auto A = [&](const double* in, double* out) { orc_skyline_multiply(n, ri, data, in, out); };
  auto M = [&](const double* in, double* out) { orc_skyline_solve(n, ri, ldlt, in, out); };
  return pcg(n, A, M, b, x, max_it, tol, iterations, matvecs, rel_res);
}

// ---------------------------------------------------------------------------
// Karhunen-Loeve expansion of the exponential kernel exp(-|x-y|/l) on
// [-A, A] (the analytic 1-D eigenproblem of Ghanem & Spanos, "Stochastic Finite
// Elements", ch. 2). The reference reads these eigen-pairs from a file
// (LognormalFileStochasticCoefficientsProvider.cs:71-118) whose format is one
// (w, l, a) row per 1-D mode and axis, a mode-index triple and an eigenvalue
// per term; the file is not shipped, so the table is rebuilt here.
//   odd 1-D index (cos modes):  c cos(wA) - w sin(wA) = 0, w in (i pi/A, (i+1/2) pi/A)
//   even 1-D index (sin modes): w cos(wA) + c sin(wA) = 0, w in ((i-1/2) pi/A, i pi/A)
//   lambda = 2c / (w^2 + c^2),  c = 1/l
//   amplitude a = 1/sqrt(A + sin(2wA)/(2w)) (cos), 1/sqrt(A - sin(2wA)/(2w)) (sin)
// ---------------------------------------------------------------------------
static double bisect(double lo, double hi, double A, double c, int is_sin) {
  auto f = [&](double w) {
    return is_sin ? (w * std::cos(w * A) + c * std::sin(w * A)) : (c * std::cos(w * A) - w * std::sin(w * A));
  };
  double flo = f(lo);
  for (int it = 0; it < 200; ++it) {
    double mid = 0.5 * (lo + hi);
    if (mid <= lo || mid >= hi) break;
    double fm = f(mid);
    if ((fm > 0) == (flo > 0)) { lo = mid; flo = fm; } else { hi = mid; }
  }
  return 0.5 * (lo + hi);
}

int orc_kl_1d_modes(double A, double l, int n, double* w, double* amp, double* lam) {
  const double pi = 3.14159265358979323846;
  double c = 1.0 / l;
  for (int k = 0; k < n; ++k) {
    int idx = k + 1;  // 1-based, as in evpPos
    int is_sin = (idx % 2 == 0);
    int i = idx / 2;  // cos: i = 0,1,2..; sin: i = 1,2,..
    double lo, hi;
    if (!is_sin) { lo = i * pi / A; hi = (i + 0.5) * pi / A; }
    else { lo = (i - 0.5) * pi / A; hi = i * pi / A; }
    double ww = bisect(lo, hi, A, c, is_sin);
    w[k] = ww;
    lam[k] = 2.0 * c / (ww * ww + c * c);
    double s = std::sin(2.0 * ww * A) / (2.0 * ww);
    amp[k] = 1.0 / std::sqrt(is_sin ? (A - s) : (A + s));
  }
  return 0;
}

// 3-D separable table: the n_terms largest products lambda_x*lambda_y*lambda_z
// over the first n1d 1-D modes per axis. Ties are broken by the 1-D index
// triple (x, then y, then z ascending) on a 2^-40-quantised eigenvalue key.
// Outputs: w3/amp3 [n_terms][3], idx3 [n_terms][3] (1-based), eig [n_terms].
int orc_kl_table(const double* L, double l, int n_terms, int n1d, double* w3, double* amp3, int* idx3,
                 double* eig) {
  std::vector<double> w[3], a[3], lam[3];
  for (int ax = 0; ax < 3; ++ax) {
    w[ax].resize(n1d); a[ax].resize(n1d); lam[ax].resize(n1d);
    orc_kl_1d_modes(0.5 * L[ax], l, n1d, w[ax].data(), a[ax].data(), lam[ax].data());
  }
  struct T { double e; int64_t q; int i, j, k; };
  std::vector<T> all;
  double emax = lam[0][0] * lam[1][0] * lam[2][0];
  for (int i = 0; i < n1d; ++i)
    for (int j = 0; j < n1d; ++j)
      for (int k = 0; k < n1d; ++k) {
        double e = (lam[0][i] * lam[1][j]) * lam[2][k];
        all.push_back({e, (int64_t)std::llround(e / emax * 1099511627776.0), i, j, k});
      }
  std::sort(all.begin(), all.end(), [](const T& x, const T& y) {
    if (x.q != y.q) return x.q > y.q;
    if (x.i != y.i) return x.i < y.i;
    if (x.j != y.j) return x.j < y.j;
    return x.k < y.k;
  });
  if ((int)all.size() < n_terms) return -1;
  for (int t = 0; t < n_terms; ++t) {
    int id[3] = {all[t].i, all[t].j, all[t].k};
    for (int ax = 0; ax < 3; ++ax) {
      w3[3 * t + ax] = w[ax][id[ax]];
      amp3[3 * t + ax] = a[ax][id[ax]];
      idx3[3 * t + ax] = id[ax] + 1;
    }
    eig[t] = all[t].e;
  }
  return 0;
}

// LognormalFileStochasticCoefficientsProvider.GetCoefficient (:173-193) with
// GetCoefficientInternal (:134-160), evaluated at the element centroid as
// Hexa8WithStochasticMaterial.GetStochasticPoints does (:112-140):
//   E = exp(mu + sum_k xi_k * sigma * sqrt(eig_k) * prod_ax amp*{cos|sin}(w*(x_ax - L_ax/2)))
//   mu = ln(mean) - sigma^2/2 (mean_correction = 1, the reference form) or ln(mean).
// Output E[n_real][n_elems].
void orc_kl_field(int ne, const double* cen, const double* L, int K, const double* w3, const double* amp3,
                  const int* idx3, const double* eig, int R, const double* xi, double mean, double sigma,
                  int mean_correction, double* E) {
  std::vector<double> psi((size_t)K * ne);
  for (int k = 0; k < K; ++k) {
    double f0 = sigma * std::sqrt(eig[k]);
    for (int e = 0; e < ne; ++e) {
      double f = f0;
      for (int ax = 0; ax < 3; ++ax) {
        double x = cen[3 * e + ax] - L[ax] / 2;
        double ww = w3[3 * k + ax], aa = amp3[3 * k + ax];
        f *= (idx3[3 * k + ax] % 2 == 0) ? aa * std::sin(ww * x) : aa * std::cos(ww * x);
      }
      psi[(size_t)k * ne + e] = f;
    }
  }
  double mu = std::log(mean) - (mean_correction ? 0.5 * sigma * sigma : 0.0);
#pragma omp parallel for schedule(static)
  for (int r = 0; r < R; ++r)
    for (int e = 0; e < ne; ++e) {
      double s = mu;
      for (int k = 0; k < K; ++k) s += xi[(size_t)r * K + k] * psi[(size_t)k * ne + e];
      E[(size_t)r * ne + e] = std::exp(s);
    }
}

// GaussianFileStochasticCoefficientsProvider (:72-108) as the Monte Carlo
// analyzer's matrix composition sees it (MonteCarloAnalyzer.cs:88-172): K_0 is
// built with coefficient 1 (order -1), K_k with GetCoefficientInternal(x, k) =
// cov * sqrt(eig_k) * prod_ax amp*{cos|sin}(w*(x_ax - L_ax/2)), and the
// realization's matrix is K_0 + sum_k xi_k K_k. The stiffness is linear in E, so
// this is one element stiffness with E = mean * (1 + sum_k xi_k * coefficient_k),
// GetCoefficient's own formula (:101-108). Output E[n_real][n_elems].
void orc_kl_field_gaussian(int ne, const double* cen, const double* L, int K, const double* w3, const double* amp3,
                           const int* idx3, const double* eig, int R, const double* xi, double mean, double cov,
                           double* E) {
  for (int r = 0; r < R; ++r)
    for (int e = 0; e < ne; ++e) {
      double result = 1;
      for (int k = 0; k < K; ++k) {
        double f = cov * std::sqrt(eig[k]);
        for (int ax = 0; ax < 3; ++ax) {
          double x = cen[3 * e + ax] - L[ax] / 2;
          double ww = w3[3 * k + ax], aa = amp3[3 * k + ax];
          f *= (idx3[3 * k + ax] % 2 == 0) ? aa * std::sin(ww * x) : aa * std::cos(ww * x);
        }
        result += xi[(size_t)r * K + k] * f;
      }
      E[(size_t)r * ne + e] = result * mean;
    }
}

// PolynomialChaosCoefficientsCalculator (PolynomialChaosCoefficientsCalculator.cs:30-300):
// basis size sum_k C(m+k-1, k), multi-indices in the reference's generation
// order (bar positions t of each total degree, advanced from the right), norms
// prod_l alpha_l!.
static double orc_fact(int f) {
  double r = 1;
  for (int i = 2; i <= f; ++i) r *= i;
  return r;
}
int orc_pc_size(int m, int p) {
  double s = 0;
  for (int k = 0; k <= p; ++k) s += orc_fact(m + k - 1) / (orc_fact(k) * orc_fact(m - 1));
  return (int)s;
}
int orc_pc_basis(int m, int p, int* basis, int* norms) {
  const int P = orc_pc_size(m, p);
  for (int i = 0; i < P * m; ++i) basis[i] = 0;
  if (m == 1) {
    for (int i = 0; i < p; ++i) basis[(i + 1) * m] = i;
  } else {
    const int mm = m - 1;
    std::vector<int> t(mm);
    int n = 0;
    for (int cur = 1; cur <= p; ++cur) {
      bool end = false, first = false;
      while (!end) {
        ++n;
        if (!first) {
          for (int i = 0; i < mm; ++i) t[i] = i + 1;
          first = true;
        } else if (t[mm - 1] < mm + cur) {
          t[mm - 1] += 1;
        } else {
          int j = mm;
          while (t[j - 1] == j + cur) --j;
          t[j - 1]++;
          for (int k = j; k < mm; ++k) t[k] = t[j - 1] + k - j + 1;
        }
        basis[n * m + 0] = t[0] - 1;
        for (int i = 1; i < mm; ++i) basis[n * m + i] = t[i] - t[i - 1] - 1;
        basis[n * m + mm] = m + cur - t[mm - 1] - 1;
        if (t[0] == cur + 1) end = true;
      }
    }
  }
  for (int k = 0; k < P; ++k) {
    int nn = 1;
    for (int j = 0; j < m; ++j) nn *= (int)orc_fact(basis[k * m + j]);
    norms[k] = nn;
  }
  return P;
}

// PolynomialChaosSolverPCGMatrixCalculator.MultiplyWithMatrix (:1062-1089), Gaussian
// branch, over m + 1 CSR matrices of one pattern (vals [m+1][nnz]): y = 0; for pos,
// for each (i, j, c) of GaussianCoefficients[pos] (PolynomialChaosCoefficientsCalculator
// .cs:294-326): y[block i] += c * K_pos u[block j]. u, y [P][n].
void orc_pc_gaussian_matvec(int n, const int64_t* rp, const int* ci, const double* vals, int64_t nnz, int m, int p,
                            const double* u, double* y) {
  const int P = orc_pc_size(m, p);
  std::vector<int> basis((size_t)P * m), norms(P);
  orc_pc_basis(m, p, basis.data(), norms.data());
  std::vector<double> tmp(n);
  for (int64_t i = 0; i < (int64_t)P * n; ++i) y[i] = 0.0;
  auto apply = [&](int pos, int i, int j, double c) {
    orc_csr_multiply(n, rp, ci, vals + (int64_t)pos * nnz, u + (int64_t)j * n, tmp.data());
    for (int r = 0; r < n; ++r) y[(int64_t)i * n + r] += c * tmp[r];
  };
  for (int i = 0; i < P; ++i) apply(0, i, i, (double)norms[i]);
  for (int v = 0; v < m; ++v)
    for (int j = 0; j < P; ++j)
      for (int k = 0; k < P; ++k) {
        bool almost = false;
        for (int l = 0; l < m; ++l)
          if (l != v && basis[j * m + l] != basis[k * m + l]) {
            almost = true;
            break;
          }
        if (almost) continue;
        if (basis[k * m + v] == basis[j * m + v] - 1)
          apply(v + 1, j, k, (double)norms[j]);
        else if (basis[k * m + v] == basis[j * m + v] + 1)
          apply(v + 1, j, k, (double)norms[j] * (basis[j * m + v] + 1));
      }
}

// One FP64 static solve of a structured nx*ny*nz block of h-cubes: element
// stiffness through the Fortran restatement with each element's E, CSR
// assembly over the free DOFs, Jacobi-PCG with SolverPCG semantics.
int orc_block_solve_pcg(int nx, int ny, int nz, double h, const uint8_t* cons, const double* Ee, double nu,
                        const double* b, double* x, int max_it, double tol, int* iterations, double* rel_res) {
  int nn = (nx + 1) * (ny + 1) * (nz + 1), ne = nx * ny * nz;
  std::vector<double> xyz(3 * (size_t)nn);
  std::vector<int> conn(8 * (size_t)ne), dof(3 * (size_t)nn);
  orc_block_nodes(nx, ny, nz, h, xyz.data());
  orc_block_conn(nx, ny, nz, conn.data());
  int N = orc_enumerate_dofs(nn, cons, dof.data());
  std::vector<double> exyz(24 * (size_t)ne), K(300 * (size_t)ne);
  for (int e = 0; e < ne; ++e)
    for (int a = 0; a < 8; ++a)
      for (int c = 0; c < 3; ++c) exyz[24 * (size_t)e + 3 * a + c] = xyz[3 * (size_t)conn[8 * e + a] + c];
  int st = 0;
  orc_h8_stiffness_batch(ne, exyz.data(), Ee, nu, K.data(), &st);
  if (st) return st;
  std::vector<int64_t> rp(N + 1);
  int64_t nnz = orc_csr_pattern(nn, ne, conn.data(), dof.data(), N, rp.data(), nullptr);
  std::vector<int> ci(nnz);
  orc_csr_pattern(nn, ne, conn.data(), dof.data(), N, rp.data(), ci.data());
  std::vector<double> v(nnz, 0.0);
  orc_csr_assemble(ne, conn.data(), dof.data(), K.data(), rp.data(), ci.data(), v.data());
  int mv = 0;
  return orc_pcg_csr_jacobi(N, rp.data(), ci.data(), v.data(), b, x, max_it, tol, iterations, &mv, rel_res);
}


/* Newmark implicit integration of a structured block, one realization.
 * NewmarkDynamicAnalyzer.cs:53-77 (coefficients a0..a7), :189-230 (RHS:
 * uu = a0 u + a2 v + a3 a, uc = a1 u + a4 v + a5 a, rhs = F + M uu + C uc),
 * :280-315 (loop over (int)(T/dt) steps, then a' = a0 (u' - u) - a2 v - a3 a,
 * v += a6 a + a7 a'); ProblemStructural.cs:138-157 (K~ = 1 K + a0 M + a1 C);
 * Hexa8.cs:403-451 (consistent mass, C_e = alpha_R M_e + beta_R K_e);
 * Hexa8.cs:512-530 + Model.cs:266-278 (inertial load: M_e times the ground
 * acceleration in DOF `acc_dir` at every element node, added to the free rows);
 * MassAccelerationSinusoidalLoad.cs:17-20 (a_g(i) = A sin(2 pi / T_p dt i)).
 * The effective matrix is factorised once (skyline LDL^T, SolverSkyline) when
 * solver == 0, or each step is solved by Jacobi PCG from x0 = 0 to `tol` when
 * solver == 1 (SolverPCG), or from the previous step's displacement when
 * solver == 2 (a starting vector only: converged to a tight `tol` the steps
 * agree with solver 1 to that tolerance, in fewer iterations).
 * tip_hist[i] = u[tip_dof] after step i. */
int orc_block_newmark(int nx, int ny, int nz, double h, const uint8_t* cons, const double* Ee, double nu, double rho,
                      double ray_alpha, double ray_beta, double nm_alpha, double nm_delta, double dt, int n_steps,
                      double acc_amp, double acc_period, int acc_dir, const double* f_static, int solver, double tol,
                      int tip_dof, double* tip_hist, double* u_final, int* total_its) {
  if (nm_delta < 0.5) return -1;
  if (nm_alpha < 0.25 * (0.5 + nm_delta) * (0.5 + nm_delta)) return -1;
  const double a0 = 1 / (nm_alpha * dt * dt), a1 = nm_delta / (nm_alpha * dt), a2 = 1 / (nm_alpha * dt);
  const double a3 = 1 / (2 * nm_alpha) - 1, a4 = nm_delta / nm_alpha - 1, a5 = dt * 0.5 * (nm_delta / nm_alpha - 2);
  const double a6 = dt * (1 - nm_delta), a7 = nm_delta * dt;
  const int nn = (nx + 1) * (ny + 1) * (nz + 1), ne = nx * ny * nz;
  std::vector<double> xyz(3 * (size_t)nn);
  std::vector<int> conn(8 * (size_t)ne), dof(3 * (size_t)nn);
  orc_block_nodes(nx, ny, nz, h, xyz.data());
  orc_block_conn(nx, ny, nz, conn.data());
  const int N = orc_enumerate_dofs(nn, cons, dof.data());
  std::vector<double> exyz(24 * (size_t)ne), K(300 * (size_t)ne), M(300 * (size_t)ne), C(300 * (size_t)ne),
      Kt(300 * (size_t)ne);
  for (int e = 0; e < ne; ++e)
    for (int a = 0; a < 8; ++a)
      for (int c = 0; c < 3; ++c) exyz[24 * (size_t)e + 3 * a + c] = xyz[3 * (size_t)conn[8 * e + a] + c];
  int st = 0;
  orc_h8_stiffness_batch(ne, exyz.data(), Ee, nu, K.data(), &st);
  if (st) return st;
  for (int e = 0; e < ne; ++e) {
    st = orc_h8_consistent_mass(&exyz[24 * (size_t)e], rho, &M[300 * (size_t)e]);
    if (st) return st;
    for (int i = 0; i < 300; ++i) {
      const size_t k = 300 * (size_t)e + i;
      C[k] = ray_alpha * M[k] + ray_beta * K[k];
      Kt[k] = 1.0 * K[k] + a0 * M[k] + a1 * C[k];
    }
  }
  // assembled M, C (products) and K~ (solve)
  std::vector<int64_t> rp(N + 1);
  const int64_t nnz = orc_csr_pattern(nn, ne, conn.data(), dof.data(), N, rp.data(), nullptr);
  std::vector<int> ci(nnz);
  orc_csr_pattern(nn, ne, conn.data(), dof.data(), N, rp.data(), ci.data());
  std::vector<double> Mv(nnz, 0.0), Cv(nnz, 0.0), Ktv(nnz, 0.0);
  orc_csr_assemble(ne, conn.data(), dof.data(), M.data(), rp.data(), ci.data(), Mv.data());
  orc_csr_assemble(ne, conn.data(), dof.data(), C.data(), rp.data(), ci.data(), Cv.data());
  std::vector<int64_t> ri;
  std::vector<double> sky;
  if (solver == 0) {
    ri.resize(N + 1);
    const int64_t len = orc_skyline_rowindex(ne, conn.data(), dof.data(), N, ri.data());
    sky.assign(len, 0.0);
    orc_skyline_assemble(ne, conn.data(), dof.data(), Kt.data(), ri.data(), sky.data());
    int zems = 0;
    st = orc_skyline_factorize(N, ri.data(), sky.data(), 1e-8, &zems);
    if (st) return st;
  } else {
    orc_csr_assemble(ne, conn.data(), dof.data(), Kt.data(), rp.data(), ci.data(), Ktv.data());
  }
  // inertial load pattern: sum_e M_e * (unit acceleration in acc_dir at all 8 nodes), free rows only
  std::vector<double> fM(N, 0.0);
  for (int e = 0; e < ne; ++e)
    for (int a = 0; a < 8; ++a)
      for (int c = 0; c < 3; ++c) {
        const int row = dof[3 * (size_t)conn[8 * e + a] + c];
        if (row < 0) continue;
        double s = 0;
        for (int b = 0; b < 8; ++b) {
          const int i = 3 * a + c, j = 3 * b + acc_dir;
          const int r0 = i < j ? i : j, c0 = i < j ? j : i;
          s += M[300 * (size_t)e + r0 * (47 - r0) / 2 + c0];
        }
        fM[row] += s;
      }
  std::vector<double> u(N, 0.0), v(N, 0.0), acc(N, 0.0), uu(N), uc(N), um(N), ucm(N), rhs(N), x(N);
  const double two_pi = 2.0 * 3.14159265358979323846;
  int its_sum = 0;
  for (int i = 0; i < n_steps; ++i) {
    const double ag = acc_amp * std::sin(two_pi / acc_period * dt * i);
    for (int k = 0; k < N; ++k) {
      uu[k] = a0 * u[k] + a2 * v[k] + a3 * acc[k];
      uc[k] = a1 * u[k] + a4 * v[k] + a5 * acc[k];
    }
    orc_csr_multiply(N, rp.data(), ci.data(), Mv.data(), uu.data(), um.data());
    orc_csr_multiply(N, rp.data(), ci.data(), Cv.data(), uc.data(), ucm.data());
    for (int k = 0; k < N; ++k) rhs[k] = (f_static ? f_static[k] : 0.0) + ag * fM[k] + um[k] + ucm[k];
    if (solver == 0) {
      orc_skyline_solve(N, ri.data(), sky.data(), rhs.data(), x.data());
    } else {
      int it = 0, mv = 0;
      double rr = 0;
      if (solver == 1) {
        std::fill(x.begin(), x.end(), 0.0);
        st = orc_pcg_csr_jacobi(N, rp.data(), ci.data(), Ktv.data(), rhs.data(), x.data(), 100000, tol, &it, &mv,
                                &rr);
      } else {
        // warm start: solve K~ dx = rhs - K~ u for the increment from zero, to the
        // same absolute stopping point ||r|| < tol ||rhs||, then x = u + dx
        orc_csr_multiply(N, rp.data(), ci.data(), Ktv.data(), u.data(), um.data());
        double nb = 0, nr = 0;
        for (int k = 0; k < N; ++k) {
          ucm[k] = rhs[k] - um[k];
          nb += rhs[k] * rhs[k];
          nr += ucm[k] * ucm[k];
        }
        std::fill(x.begin(), x.end(), 0.0);
        if (nr > 0) {
          const double tol_inc = nb > 0 ? tol * std::sqrt(nb / nr) : tol;
          st = orc_pcg_csr_jacobi(N, rp.data(), ci.data(), Ktv.data(), ucm.data(), x.data(), 100000, tol_inc, &it,
                                  &mv, &rr);
        }
        for (int k = 0; k < N; ++k) x[k] += u[k];
      }
      if (st) return st;
      its_sum += it;
    }
    for (int k = 0; k < N; ++k) {
      const double an = a0 * (x[k] - u[k]) - a2 * v[k] - a3 * acc[k];
      v[k] += a6 * acc[k] + a7 * an;
      acc[k] = an;
      u[k] = x[k];
    }
    if (tip_hist) tip_hist[i] = (tip_dof >= 0 && tip_dof < N) ? u[tip_dof] : 0.0;
  }
  if (u_final) std::copy(u.begin(), u.end(), u_final);
  if (total_its) *total_its = its_sum;
  return 0;
}


/* Realizations in parallel: one realization per OpenMP thread, each solved as
 * orc_block_solve_pcg does (its inner OpenMP loops run on that one thread).
 * E [R][ne], b shared, x [R][N]; status/iterations/rel_res per realization. */
void orc_block_solve_pcg_batch(int R, int nx, int ny, int nz, double h, const uint8_t* cons, const double* E, double nu,
                               const double* b, double* x, int N, int max_it, double tol, int* status,
                               int* iterations, double* rel_res) {
  const int64_t ne = (int64_t)nx * ny * nz;
#pragma omp parallel for schedule(dynamic, 1)
  for (int r = 0; r < R; ++r)
    status[r] = orc_block_solve_pcg(nx, ny, nz, h, cons, E + r * ne, nu, b, x + (int64_t)r * N, max_it, tol,
                                    &iterations[r], &rel_res[r]);
}

/* orc_block_newmark for R realizations in parallel (one per OpenMP thread).
 * E [R][ne]; tip_hist [R][n_steps]; u_final [R][N]; per-realization status and
 * total iterations. */
void orc_block_newmark_batch(int R, int nx, int ny, int nz, double h, const uint8_t* cons, const double* E, double nu,
                             double rho, double ray_alpha, double ray_beta, double nm_alpha, double nm_delta,
                             double dt, int n_steps, double acc_amp, double acc_period, int acc_dir,
                             const double* f_static, int solver, double tol, int tip_dof, int N, double* tip_hist,
                             double* u_final, int* total_its, int* status) {
  const int64_t ne = (int64_t)nx * ny * nz;
#pragma omp parallel for schedule(dynamic, 1)
  for (int r = 0; r < R; ++r)
    status[r] = orc_block_newmark(nx, ny, nz, h, cons, E + r * ne, nu, rho, ray_alpha, ray_beta, nm_alpha, nm_delta,
                                  dt, n_steps, acc_amp, acc_period, acc_dir, f_static, solver, tol, tip_dof,
                                  tip_hist + (int64_t)r * n_steps, u_final + (int64_t)r * N, &total_its[r]);
}

}  // extern "C"
