// Batched Hexa8 element kernels (FP64): stiffness K_e = sum_gp w B^T D B and
// consistent mass, the device twins of CalcH8GaussMatrices + CalcH8K
// (FEMElements/FEMElements/rElHexa8.f90:422-464, 489-543) and
// Hexa8.CalculateConsistentMass (ISAAR.MSolve.PreProcessor/Elements/Hexa8.cs:403-435).
//
// One CTA handles 8 elements. Phase 1: 64 threads, one per (element, Gauss
// point), compute the shape-function natural derivatives, the Jacobian, its
// determinant and inverse, the Cartesian derivatives dN/dx (the nonzeros of
// B) and the weight, into shared memory. Phase 2: all threads produce the 300
// packed entries of each element, each entry summed over the 8 Gauss points
// in the reference's order (xi outer, zeta inner). Output writes are
// contiguous across threads.
#include "msg_internal.h"

namespace msg {
namespace {

constexpr int kEPB = 8;      // elements per CTA
constexpr int kThreads = 256;

__constant__ unsigned short c_pair_i[300];
__constant__ unsigned short c_pair_j[300];

struct GaussData {
  double dx[kEPB][8][8][3];  // [elem][gp][node][x,y,z] = dN_node/dx_c
  double w[kEPB][8];
  double S[8][8];            // shape values [gp][node] (same for every element)
};

// rElHexa8.f90:435-445 literal 2-point rule.
__device__ __forceinline__ double gauss_pt(int i) { return i ? .5773502691896 : -.5773502691896; }

__device__ void gauss_point(const double* __restrict__ xyz, int gp, double* dxyz /*[8][3]*/, double* w,
                            double* S8, int* status) {
  const int ix = gp >> 2, iy = (gp >> 1) & 1, iz = gp & 1;
  const double xi = gauss_pt(ix), eta = gauss_pt(iy), zeta = gauss_pt(iz);
  // CalcH8NablaShape (:25-69)
  const double s = 0.35355339059327376220042218105242;
  const double xp = (1.0 + xi) * s, ep = (1.0 + eta) * s, zp = (1.0 + zeta) * s;
  const double xm = (1.0 - xi) * s, em = (1.0 - eta) * s, zm = (1.0 - zeta) * s;
  double ds[24];
  ds[0] = -(em * zm); ds[1] = -ds[0]; ds[2] = ep * zm; ds[3] = -ds[2];
  ds[4] = -(em * zp); ds[5] = -ds[4]; ds[6] = ep * zp; ds[7] = -ds[6];
  ds[8] = -(xm * zm); ds[9] = -(xp * zm); ds[10] = -ds[9]; ds[11] = -ds[8];
  ds[12] = -(xm * zp); ds[13] = -(xp * zp); ds[14] = -ds[13]; ds[15] = -ds[12];
  ds[16] = -(xm * em); ds[17] = -(xp * em); ds[18] = -(xp * ep); ds[19] = -(xm * ep);
  ds[20] = -ds[16]; ds[21] = -ds[17]; ds[22] = -ds[18]; ds[23] = -ds[19];
  // CalcH8JDetJ (:141-208)
  double J[9];
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      double acc = ds[8 * a] * xyz[i];
#pragma unroll
      for (int n = 1; n < 8; ++n) acc = acc + ds[8 * a + n] * xyz[3 * n + i];
      J[3 * a + i] = acc;
    }
  const double d1 = J[0] * (J[4] * J[8] - J[7] * J[5]);
  const double d2 = -J[1] * (J[3] * J[8] - J[6] * J[5]);
  const double d3 = J[2] * (J[3] * J[7] - J[6] * J[4]);
  const double det = d1 + d2 + d3;
  if (det < 0.00000001) atomicMin(status, MSG_ERR_NEG_DET);
  // CalcH8B inverse (:232-250)
  const double inv = 1.0 / det;
  double Ji[9];
  Ji[0] = (J[4] * J[8] - J[7] * J[5]) * inv;
  Ji[3] = (J[6] * J[5] - J[3] * J[8]) * inv;
  Ji[6] = (J[3] * J[7] - J[6] * J[4]) * inv;
  Ji[1] = (J[7] * J[2] - J[1] * J[8]) * inv;
  Ji[4] = (J[0] * J[8] - J[6] * J[2]) * inv;
  Ji[7] = (J[6] * J[1] - J[7] * J[0]) * inv;
  Ji[2] = (J[1] * J[5] - J[4] * J[2]) * inv;
  Ji[5] = (J[3] * J[2] - J[0] * J[5]) * inv;
  Ji[8] = (J[0] * J[4] - J[3] * J[1]) * inv;
#pragma unroll
  for (int n = 0; n < 8; ++n) {
    dxyz[3 * n + 0] = Ji[0] * ds[n] + Ji[1] * ds[8 + n] + Ji[2] * ds[16 + n];
    dxyz[3 * n + 1] = Ji[3] * ds[n] + Ji[4] * ds[8 + n] + Ji[5] * ds[16 + n];
    dxyz[3 * n + 2] = Ji[6] * ds[n] + Ji[7] * ds[8 + n] + Ji[8] * ds[16 + n];
  }
  *w = 1.0 * 1.0 * 1.0 * det;
  if (S8) {  // CalcH8Shape (:93-117)
    const double c = 0.5;
    const double Xp = (1.0 + xi) * c, Ep = (1.0 + eta) * c, Zp = (1.0 + zeta) * c;
    const double Xm = (1.0 - xi) * c, Em = (1.0 - eta) * c, Zm = (1.0 - zeta) * c;
    S8[0] = Xm * Em * Zm; S8[1] = Xp * Em * Zm; S8[2] = Xp * Ep * Zm; S8[3] = Xm * Ep * Zm;
    S8[4] = Xm * Em * Zp; S8[5] = Xp * Em * Zp; S8[6] = Xp * Ep * Zp; S8[7] = Xm * Ep * Zp;
  }
}

// Column i of B (6 strains) from dN/dx of node a = i/3, component c = i%3
// (rElHexa8.f90:253-396: rows exx, eyy, ezz, gxy, gyz, gzx).
__device__ __forceinline__ void b_column(const double* d /*dN_a/dx[3]*/, int c, double* B6) {
  B6[0] = c == 0 ? d[0] : 0.0;
  B6[1] = c == 1 ? d[1] : 0.0;
  B6[2] = c == 2 ? d[2] : 0.0;
  B6[3] = c == 0 ? d[1] : (c == 1 ? d[0] : 0.0);
  B6[4] = c == 1 ? d[2] : (c == 2 ? d[1] : 0.0);
  B6[5] = c == 0 ? d[2] : (c == 2 ? d[0] : 0.0);
}

__global__ void __launch_bounds__(kThreads) k_h8_ke(int n, const double* __restrict__ xyz,
                                                    const double* __restrict__ Ev, double E_scalar, double nu,
                                                    double* __restrict__ K, int* __restrict__ status) {
  __shared__ GaussData g;
  __shared__ double sD[kEPB][3];  // e3 (diag), e2 (off), e4 (shear) per element
  const int e0 = blockIdx.x * kEPB;
  const int t = threadIdx.x;
  if (t < kEPB * 8) {
    const int le = t >> 3, gp = t & 7, e = e0 + le;
    if (e < n) {
      double x[24];
#pragma unroll
      for (int k = 0; k < 24; ++k) x[k] = xyz[(size_t)e * 24 + k];
      gauss_point(x, gp, &g.dx[le][gp][0][0], &g.w[le][gp], nullptr, status);
    }
  } else if (t < kEPB * 8 + kEPB) {
    const int le = t - kEPB * 8, e = e0 + le;
    if (e < n) {  // ElasticMaterial3D.GetConstitutiveMatrix (:20-44)
      const double E = Ev ? Ev[e] : E_scalar;
      const double e1 = E / (1.0 + nu);
      const double e2 = e1 * nu / (1.0 - 2.0 * nu);
      sD[le][0] = e1 + e2;
      sD[le][1] = e2;
      sD[le][2] = e1 * 0.5;
    }
  }
  __syncthreads();
  for (int q = t; q < kEPB * 300; q += kThreads) {
    const int le = q / 300, idx = q - le * 300, e = e0 + le;
    if (e >= n) break;
    const int i = c_pair_i[idx], j = c_pair_j[idx];
    const int a = i / 3, ci = i - 3 * a, b = j / 3, cj = j - 3 * b;
    const double d3 = sD[le][0], d2 = sD[le][1], d4 = sD[le][2];
    double acc = 0.0;
#pragma unroll 1
    for (int gp = 0; gp < 8; ++gp) {
      double Bi[6], Bj[6];
      b_column(g.dx[le][gp][a], ci, Bi);
      b_column(g.dx[le][gp][b], cj, Bj);
      // eb = D B_i with the isotropic D (rows summed left to right as CalcH8K :514-531)
      double eb[6];
      eb[0] = d3 * Bi[0] + d2 * Bi[1] + d2 * Bi[2];
      eb[1] = d2 * Bi[0] + d3 * Bi[1] + d2 * Bi[2];
      eb[2] = d2 * Bi[0] + d2 * Bi[1] + d3 * Bi[2];
      eb[3] = d4 * Bi[3];
      eb[4] = d4 * Bi[4];
      eb[5] = d4 * Bi[5];
      double st = Bj[0] * eb[0] + Bj[1] * eb[1] + Bj[2] * eb[2] + Bj[3] * eb[3] + Bj[4] * eb[4] + Bj[5] * eb[5];
      acc = acc + st * g.w[le][gp];
    }
    K[(size_t)e * 300 + idx] = acc;
  }
}

__global__ void __launch_bounds__(kThreads) k_h8_me(int n, const double* __restrict__ xyz, double rho,
                                                    double* __restrict__ M, int* __restrict__ status) {
  __shared__ GaussData g;
  const int e0 = blockIdx.x * kEPB;
  const int t = threadIdx.x;
  if (t < kEPB * 8) {
    const int le = t >> 3, gp = t & 7, e = e0 + le;
    if (e < n) {
      double x[24];
#pragma unroll
      for (int k = 0; k < 24; ++k) x[k] = xyz[(size_t)e * 24 + k];
      double S8[8];
      gauss_point(x, gp, &g.dx[le][gp][0][0], &g.w[le][gp], S8, status);
      if (le == 0)
        for (int k = 0; k < 8; ++k) g.S[gp][k] = S8[k];
    }
  }
  __syncthreads();
  for (int q = t; q < kEPB * 300; q += kThreads) {
    const int le = q / 300, idx = q - le * 300, e = e0 + le;
    if (e >= n) break;
    const int i = c_pair_i[idx], j = c_pair_j[idx];
    const int a = i / 3, ci = i - 3 * a, b = j / 3, cj = j - 3 * b;
    double acc = 0.0;
    if (ci == cj) {
      for (int gp = 0; gp < 8; ++gp) acc = acc + g.S[gp][a] * g.S[gp][b] * (g.w[le][gp] * rho);
    }
    M[(size_t)e * 300 + idx] = acc;
  }
}

// Strain / stress recovery and internal forces of a batch of element
// instances (an instance = one element of one realization), the device twin
// of Hexa8.CalculateStresses + CalculateForces (ISAAR.MSolve.PreProcessor/
// Elements/Hexa8.cs:453-510) over CalcH8Strains and CalcH8Forces
// (FEMElements/FEMElements/rElHexa8.f90:636-648, 724-747) with the elastic
// material update (ElasticMaterial3D.cs:20-44, 75-81: the stored strain is the
// increment, stresses = D * increment). Per Gauss point m: strains = B_m u,
// stresses = D(E) B_m du; forces = sum_m w_m B_m^T stresses_m. Sums follow the
// reference's order (24 columns of B; 6 columns of D; 6 rows of B^T; Gauss
// points xi outer, zeta inner). The displacements come from an instance array
// u [n][24] or are gathered from a realization batch X [R][n_dofs] through
// the connectivity and the DOF map (constrained DOFs: 0).
struct StressIn {
  const double* xyz;   // [n_e][24]
  const double* E;     // [n] or nullptr (E_scalar)
  double E_scalar, nu;
  const double* u;     // [n][24] or nullptr (gather from X)
  const double* du;    // [n][24] or nullptr (du = u)
  const double* X;     // [R][n_dofs]
  const int* conn;     // [n_e][8]
  const int* dof;      // [n_nodes][3]
  int n_e, n_dofs;
};

struct StressShared {
  double dx[kEPB][8][8][3];
  double w[kEPB][8];
  double sig[kEPB][8][6];
};

__global__ void __launch_bounds__(kThreads) k_h8_stress(int n, StressIn in, double* __restrict__ strains,
                                                        double* __restrict__ stresses, double* __restrict__ forces,
                                                        int* __restrict__ status) {
  __shared__ StressShared g;
  const int i0 = blockIdx.x * kEPB;
  const int t = threadIdx.x;
  if (t < kEPB * 8) {
    const int le = t >> 3, gp = t & 7, i = i0 + le;
    if (i < n) {
      const int e = i % in.n_e;
      const size_t r = (size_t)(i / in.n_e);
      double x[24];
#pragma unroll
      for (int k = 0; k < 24; ++k) x[k] = in.xyz[(size_t)e * 24 + k];
      gauss_point(x, gp, &g.dx[le][gp][0][0], &g.w[le][gp], nullptr, status);
      double u[24], du[24];
      if (in.u) {
#pragma unroll
        for (int k = 0; k < 24; ++k) u[k] = in.u[(size_t)i * 24 + k];
      } else {
#pragma unroll
        for (int a = 0; a < 8; ++a) {
          const int node = in.conn[(size_t)e * 8 + a];
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            const int d = in.dof[(size_t)node * 3 + c];
            u[3 * a + c] = d >= 0 ? in.X[r * in.n_dofs + d] : 0.0;
          }
        }
      }
      if (in.du) {
#pragma unroll
        for (int k = 0; k < 24; ++k) du[k] = in.du[(size_t)i * 24 + k];
      } else {
#pragma unroll
        for (int k = 0; k < 24; ++k) du[k] = u[k];
      }
      const double* dx = &g.dx[le][gp][0][0];
      // CalcH8Strains: MatMul(B, u) row by row over the 24 columns
      double eps[6], deps[6];
#pragma unroll
      for (int row = 0; row < 6; ++row) {
        double s = 0.0, sd = 0.0;
#pragma unroll
        for (int col = 0; col < 24; ++col) {
          double B6[6];
          b_column(dx + 3 * (col / 3), col % 3, B6);
          s = s + B6[row] * u[col];
          sd = sd + B6[row] * du[col];
        }
        eps[row] = s;
        deps[row] = sd;
      }
      // ElasticMaterial3D: stresses = D * (strain increment), row by row over 6 columns
      const double E = in.E ? in.E[i] : in.E_scalar;
      const double e1 = E / (1.0 + in.nu);
      const double e2 = e1 * in.nu / (1.0 - 2.0 * in.nu);
      const double D[6][6] = {{e1 + e2, e2, e2, 0, 0, 0}, {e2, e1 + e2, e2, 0, 0, 0}, {e2, e2, e1 + e2, 0, 0, 0},
                              {0, 0, 0, e1 * 0.5, 0, 0},   {0, 0, 0, 0, e1 * 0.5, 0},   {0, 0, 0, 0, 0, e1 * 0.5}};
      double sig[6];
#pragma unroll
      for (int row = 0; row < 6; ++row) {
        double s = 0.0;
#pragma unroll
        for (int col = 0; col < 6; ++col) s = s + D[row][col] * deps[col];
        sig[row] = s;
        g.sig[le][gp][row] = s;
      }
      if (strains)
#pragma unroll
        for (int row = 0; row < 6; ++row) strains[((size_t)i * 8 + gp) * 6 + row] = eps[row];
      if (stresses)
#pragma unroll
        for (int row = 0; row < 6; ++row) stresses[((size_t)i * 8 + gp) * 6 + row] = sig[row];
    }
  }
  __syncthreads();
  if (!forces) return;
  // CalcH8Forces: forces = forces + w_m * MatMul(Transpose(B_m), stresses_m), m in Gauss order
  for (int q = t; q < kEPB * 24; q += kThreads) {
    const int le = q / 24, col = q - le * 24, i = i0 + le;
    if (i >= n) break;
    double f = 0.0;
#pragma unroll 1
    for (int gp = 0; gp < 8; ++gp) {
      double B6[6];
      b_column(&g.dx[le][gp][col / 3][0], col % 3, B6);
      double s = 0.0;
#pragma unroll
      for (int row = 0; row < 6; ++row) s = s + B6[row] * g.sig[le][gp][row];
      f = f + g.w[le][gp] * s;
    }
    forces[(size_t)i * 24 + col] = f;
  }
}

bool g_pairs_ready[64] = {false};
std::mutex g_pairs_mu;

int ensure_pairs(Context* ctx) {
  std::lock_guard<std::mutex> lk(g_pairs_mu);
  if (ctx->device >= 0 && ctx->device < 64 && g_pairs_ready[ctx->device]) return MSG_OK;
  unsigned short pi[300], pj[300];
  int k = 0;
  for (int i = 0; i < 24; ++i)
    for (int j = i; j < 24; ++j) { pi[k] = (unsigned short)i; pj[k] = (unsigned short)j; ++k; }
  MSG_CUDA(ctx, cudaMemcpyToSymbol(c_pair_i, pi, sizeof(pi)));
  MSG_CUDA(ctx, cudaMemcpyToSymbol(c_pair_j, pj, sizeof(pj)));
  if (ctx->device >= 0 && ctx->device < 64) g_pairs_ready[ctx->device] = true;
  return MSG_OK;
}

}  // namespace

int launch_h8_ke(Context* ctx, int n, const double* d_xyz, const double* d_E, double E_scalar, double nu,
                 double* d_K, int* d_status) {
  if (n <= 0) return MSG_OK;
  MSG_TRY(ensure_pairs(ctx));
  k_h8_ke<<<(n + kEPB - 1) / kEPB, kThreads, 0, ctx->stream>>>(n, d_xyz, d_E, E_scalar, nu, d_K, d_status);
  count_launch(ctx);
  MSG_CUDA(ctx, cudaGetLastError());
  return MSG_OK;
}

int launch_h8_stress(Context* ctx, int n, const double* d_xyz, const double* d_E, double E_scalar, double nu,
                     const double* d_u, const double* d_du, const double* d_X, const int* d_conn, const int* d_dof,
                     int n_e, int n_dofs, double* d_strains, double* d_stresses, double* d_forces, int* d_status) {
  if (n <= 0) return MSG_OK;
  StressIn in{d_xyz, d_E, E_scalar, nu, d_u, d_du, d_X, d_conn, d_dof, n_e, n_dofs};
  k_h8_stress<<<(n + kEPB - 1) / kEPB, kThreads, 0, ctx->stream>>>(n, in, d_strains, d_stresses, d_forces,
                                                                   d_status);
  count_launch(ctx);
  MSG_CUDA(ctx, cudaGetLastError());
  return MSG_OK;
}

int launch_h8_me(Context* ctx, int n, const double* d_xyz, double rho, double* d_M, int* d_status) {
  if (n <= 0) return MSG_OK;
  MSG_TRY(ensure_pairs(ctx));
  k_h8_me<<<(n + kEPB - 1) / kEPB, kThreads, 0, ctx->stream>>>(n, d_xyz, rho, d_M, d_status);
  count_launch(ctx);
  MSG_CUDA(ctx, cudaGetLastError());
  return MSG_OK;
}

}  // namespace msg
