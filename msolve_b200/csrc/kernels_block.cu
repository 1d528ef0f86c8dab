// Batched mixed-precision Monte Carlo solve on a structured cube lattice.
//
// The path of MonteCarloAnalyzerWithStochasticMaterial.SolveNormal
// (ISAAR.MSolve.Analyzers/MonteCarloAnalyzerWithStochasticMaterial.cs:232-296),
// restated for all realizations at once. For a lattice of equal cubes every
// element stiffness is K_e = E_e * Khat (Hexa8WithStochasticMaterial.cs:61-110
// evaluates E once at the centroid), so the global operator is applied
// matrix-free: y_n = sum_{e owns n} E_e * Khat[rows of n] . u_e.
//
// Layout (realization innermost): a vector of the batch is
// v[(node*3 + comp)*Rp + r], node = i + NX*(j + NY*k) in generator order,
// r = realization. A warp is 32 realizations of one node; every load and store
// of the stencil is one coalesced 128-byte line, and per-realization dot
// products need no cross-lane reduction.
//
// Operator kernel: one warp walks a pencil of nodes along x (fixed j,k),
// keeping a 3x3x3-node window of the input vector and the 2x2x2 elements
// around the current node in registers; each step loads one new 3x3 plane and
// produces the node's 3 outputs with 8 x (8 x 9) fused multiply-adds against
// Khat (a __grid_constant__ kernel parameter, so every Khat operand is a
// warp-uniform constant-bank read). Each output is written exactly once: no
// atomics, results are deterministic and independent of the batch mix.
//
// Solver: iterative refinement. Outer step (FP64): x += d, r = b - K x with the
// FP64 operator, ||r||/||b|| < tol ends the realization. Inner solve (FP32):
// Jacobi-PCG on K d = r to a relative residual eta with the FP32 operator:
//   k_inner_op : p_new = dinv.r + beta p_old (window), q = K p_new, partial p.q
//   k_alpha    : alpha = (z.r)/(p.q) per realization (fixed-order sum)
//   k_update   : d += alpha p_new, r -= alpha q, partials (dinv r).r and r.r
//   k_beta     : beta, inner convergence, count of active realizations
// The inner loop is captured as a CUDA graph of kChunk iterations; the host
// reads the active count after each chunk.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "msg_internal.h"

namespace msg {
namespace {

constexpr int kTJ = 2, kTK = 2, kWarps = kTJ * kTK;  // pencils per CTA (2 x 2 in (j,k))

struct KhatF { float k[576]; };
struct KhatD { double k[576]; };

struct Lattice {
  int NX, NY, NZ;     // nodes per axis
  int nx, ny, nz;     // elements per axis
  int Rp;             // padded realizations (multiple of 32)
  int tiles_j;        // ceil(NY / kTJ)
};

template <class T> struct KhatOf;
template <> struct KhatOf<float> { using type = KhatF; };
template <> struct KhatOf<double> { using type = KhatD; };

// Node-centric stencil along one pencil. Loader(node, out3) fills the 3
// components of the operator input at `node` (called for in-range nodes only);
// Emit(i, node, own3, y3) consumes the centre value and K*own at node i.
template <class T, class Loader, class Emit>
__device__ __forceinline__ void pencil_sweep(const Lattice& L, const typename KhatOf<T>::type& K, int j, int k, int rr,
                                             const T* __restrict__ E, Loader load, Emit emit) {
  T W[3][3][3][3];  // [dx][dy][dz][comp], dx=0 <-> x=i-1
  T Ew[2][2][2];    // [ex][ey][ez]: element (i-1+ex, j-1+ey, k-1+ez)
  const int Rp = L.Rp;
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int dy = 0; dy < 3; ++dy)
#pragma unroll
      for (int dz = 0; dz < 3; ++dz)
#pragma unroll
        for (int c = 0; c < 3; ++c) W[a][dy][dz][c] = T(0);
  // plane x = 0 into W[1]
#pragma unroll
  for (int dy = 0; dy < 3; ++dy)
#pragma unroll
    for (int dz = 0; dz < 3; ++dz) {
      const int jj = j + dy - 1, kk = k + dz - 1;
      if (jj >= 0 && jj < L.NY && kk >= 0 && kk < L.NZ) load((jj + L.NY * kk) * L.NX + 0, W[1][dy][dz]);
    }
#pragma unroll
  for (int ey = 0; ey < 2; ++ey)
#pragma unroll
    for (int ez = 0; ez < 2; ++ez) Ew[0][ey][ez] = T(0);

#pragma unroll 1
  for (int i = 0; i < L.NX; ++i) {
    // next plane x = i+1 into W[2]
#pragma unroll
    for (int dy = 0; dy < 3; ++dy)
#pragma unroll
      for (int dz = 0; dz < 3; ++dz) {
#pragma unroll
        for (int c = 0; c < 3; ++c) W[2][dy][dz][c] = T(0);
        const int jj = j + dy - 1, kk = k + dz - 1;
        if (i + 1 < L.NX && jj >= 0 && jj < L.NY && kk >= 0 && kk < L.NZ)
          load((jj + L.NY * kk) * L.NX + i + 1, W[2][dy][dz]);
      }
    // elements with x-index i
#pragma unroll
    for (int ey = 0; ey < 2; ++ey)
#pragma unroll
      for (int ez = 0; ez < 2; ++ez) {
        const int ej = j - 1 + ey, ek = k - 1 + ez;
        T v = T(0);
        if (i < L.nx && ej >= 0 && ej < L.ny && ek >= 0 && ek < L.nz)
          v = E[(size_t)(i + L.nx * (ej + L.ny * ek)) * Rp + rr];
        Ew[1][ey][ez] = v;
      }
    // y = sum_e E_e * Khat[a_n rows] . u_e
    T y[3] = {T(0), T(0), T(0)};
#pragma unroll
    for (int ex = 0; ex < 2; ++ex)
#pragma unroll
      for (int ey = 0; ey < 2; ++ey)
#pragma unroll
        for (int ez = 0; ez < 2; ++ez) {
          const int an = corner_id(1 - ex, 1 - ey, 1 - ez);
          T t[3] = {T(0), T(0), T(0)};
#pragma unroll
          for (int bx = 0; bx < 2; ++bx)
#pragma unroll
            for (int by = 0; by < 2; ++by)
#pragma unroll
              for (int bz = 0; bz < 2; ++bz) {
                const int bn = corner_id(bx, by, bz);
#pragma unroll
                for (int c = 0; c < 3; ++c)
#pragma unroll
                  for (int c2 = 0; c2 < 3; ++c2)
                    t[c] = fma(K.k[(3 * an + c) * 24 + 3 * bn + c2], W[ex + bx][ey + by][ez + bz][c2], t[c]);
              }
#pragma unroll
          for (int c = 0; c < 3; ++c) y[c] = fma(Ew[ex][ey][ez], t[c], y[c]);
        }
    emit(i, (j + L.NY * k) * L.NX + i, W[1][1][1], y);
    // shift the window
#pragma unroll
    for (int dy = 0; dy < 3; ++dy)
#pragma unroll
      for (int dz = 0; dz < 3; ++dz)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          W[0][dy][dz][c] = W[1][dy][dz][c];
          W[1][dy][dz][c] = W[2][dy][dz][c];
        }
#pragma unroll
    for (int ey = 0; ey < 2; ++ey)
#pragma unroll
      for (int ez = 0; ez < 2; ++ez) Ew[0][ey][ez] = Ew[1][ey][ez];
  }
}

// Per-CTA reduction of per-realization partials over its warps (same lanes).
template <int NV>
__device__ __forceinline__ void cta_partial(const double (&v)[NV], double* __restrict__ out, int tile, int Rp, int rr) {
  __shared__ double sh[kWarps][NV][32];
  const int lane = threadIdx.x, w = threadIdx.y;
#pragma unroll
  for (int q = 0; q < NV; ++q) sh[w][q][lane] = v[q];
  __syncthreads();
  if (w == 0) {
#pragma unroll
    for (int q = 0; q < NV; ++q) {
      double s = 0;
#pragma unroll
      for (int ww = 0; ww < kWarps; ++ww) s += sh[ww][q][lane];
      out[((size_t)tile * Rp + rr) * NV + q] = s;
    }
  }
}

__device__ __forceinline__ void pencil_of(const Lattice& L, int& j, int& k) {
  const int tile = blockIdx.x;
  const int tj = tile % L.tiles_j, tk = tile / L.tiles_j;
  j = tj * kTJ + (threadIdx.y % kTJ);
  k = tk * kTK + (threadIdx.y / kTJ);
}

// FP32 inner operator with the fused direction update.
__global__ void __launch_bounds__(128, 4)
    k_inner_op(Lattice L, const __grid_constant__ KhatF K, const float* __restrict__ r, const float* __restrict__ pold,
               float* __restrict__ pnew, const float* __restrict__ dinv, const float* __restrict__ E,
               const uint8_t* __restrict__ mask, const float* __restrict__ beta, float* __restrict__ q,
               double* __restrict__ partial) {
  int j, k;
  pencil_of(L, j, k);
  const int Rp = L.Rp;
  const int rr = blockIdx.y * 32 + threadIdx.x;
  const float b = beta[rr];
  double pq[1] = {0.0};
  if (j < L.NY && k < L.NZ) {
    auto load = [&](int node, float* o) {
      const float dv = dinv[(size_t)node * Rp + rr];
      const size_t base = (size_t)node * 3 * Rp + rr;
#pragma unroll
      for (int c = 0; c < 3; ++c) o[c] = fmaf(dv, r[base + c * Rp], b * pold[base + c * Rp]);
    };
    auto emit = [&](int, int node, const float* own, const float* y) {
      const uint8_t m = mask[node];
      const size_t base = (size_t)node * 3 * Rp + rr;
      float acc = 0.f;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const float qc = ((m >> c) & 1) ? 0.f : y[c];
        pnew[base + c * Rp] = own[c];
        q[base + c * Rp] = qc;
        acc = fmaf(own[c], qc, acc);
      }
      pq[0] += (double)acc;
    };
    pencil_sweep<float>(L, K, j, k, rr, E, load, emit);
  }
  cta_partial<1>(pq, partial, blockIdx.x, Rp, rr);
}

// FP64 refinement step: x_new = x_old + d (window), r = b - K x_new (own node),
// r32 = (float) r; partials ||r||^2 and (dinv r32).r32.
__global__ void __launch_bounds__(128)
    k_resid_op(Lattice L, const __grid_constant__ KhatD K, const double* __restrict__ xold,
               const float* __restrict__ d, double* __restrict__ xnew, const double* __restrict__ b_lat,
               const double* __restrict__ E, const uint8_t* __restrict__ mask, const float* __restrict__ dinv,
               float* __restrict__ r32, double* __restrict__ partial) {
  int j, k;
  pencil_of(L, j, k);
  const int Rp = L.Rp;
  const int rr = blockIdx.y * 32 + threadIdx.x;
  double acc[2] = {0.0, 0.0};
  if (j < L.NY && k < L.NZ) {
    auto load = [&](int node, double* o) {
      const size_t base = (size_t)node * 3 * Rp + rr;
#pragma unroll
      for (int c = 0; c < 3; ++c) o[c] = xold[base + c * Rp] + (double)d[base + c * Rp];
    };
    auto emit = [&](int, int node, const double* own, const double* y) {
      const uint8_t m = mask[node];
      const size_t base = (size_t)node * 3 * Rp + rr;
      const double dv = (double)dinv[(size_t)node * Rp + rr];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const double rc = ((m >> c) & 1) ? 0.0 : b_lat[node * 3 + c] - y[c];
        xnew[base + c * Rp] = own[c];
        const float rf = (float)rc;
        r32[base + c * Rp] = rf;
        acc[0] += rc * rc;
        acc[1] += dv * (double)rf * (double)rf;
      }
    };
    pencil_sweep<double>(L, K, j, k, rr, E, load, emit);
  }
  cta_partial<2>(acc, partial, blockIdx.x, Rp, rr);
}

// Jacobi diagonal: K_nn,cc = Khat_diag * sum of E over the node's elements
// (all 24 diagonal entries of a cube's Khat are equal).
__global__ void k_dinv(Lattice L, double kdiag, const float* __restrict__ E, float* __restrict__ dinv) {
  const int node = blockIdx.x;
  const int i = node % L.NX, j = (node / L.NX) % L.NY, k = node / (L.NX * L.NY);
  for (int rr = threadIdx.x; rr < L.Rp; rr += blockDim.x) {
    double s = 0;
    for (int ez = -1; ez <= 0; ++ez)
      for (int ey = -1; ey <= 0; ++ey)
        for (int ex = -1; ex <= 0; ++ex) {
          const int ei = i + ex, ej = j + ey, ek = k + ez;
          if (ei >= 0 && ei < L.nx && ej >= 0 && ej < L.ny && ek >= 0 && ek < L.nz)
            s += (double)E[(size_t)(ei + L.nx * (ej + L.ny * ek)) * L.Rp + rr];
        }
    dinv[(size_t)node * L.Rp + rr] = (float)(1.0 / (kdiag * s));
  }
}

// d += alpha p, r -= alpha q; partials (dinv r).r and r.r per realization.
// Thread = one float4 of realizations; G node groups per CTA when Rp/4 < 256.
__global__ void __launch_bounds__(256) k_update(int n_nodes, int Rp, const float* __restrict__ alpha,
                                                const float* __restrict__ p, const float* __restrict__ q,
                                                float* __restrict__ d, float* __restrict__ r,
                                                const float* __restrict__ dinv, double* __restrict__ partial) {
  const int Q = Rp >> 2;
  const int t = threadIdx.x;
  const int G = Q >= 256 ? 1 : 256 / Q;
  const int g = Q >= 256 ? 0 : t / Q;
  const int nodes_per_blk = (n_nodes + gridDim.x - 1) / gridDim.x;
  const int n0 = blockIdx.x * nodes_per_blk, n1 = min(n_nodes, n0 + nodes_per_blk);
  extern __shared__ double sh[];  // [G][Q][8] when G > 1
  for (int qb = (Q >= 256 ? t : t % Q); qb < Q && (Q >= 256 || t < G * Q); qb += (Q >= 256 ? 256 : Q)) {
    const float4 a4 = reinterpret_cast<const float4*>(alpha)[qb];
    double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int n = n0 + g; n < n1; n += G) {
      const float4 dv = reinterpret_cast<const float4*>(dinv + (size_t)n * Rp)[qb];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const size_t o = ((size_t)n * 3 + c) * Rp;
        const float4 pv = reinterpret_cast<const float4*>(p + o)[qb];
        const float4 qv = reinterpret_cast<const float4*>(q + o)[qb];
        float4 dd = reinterpret_cast<const float4*>(d + o)[qb];
        float4 rv = reinterpret_cast<const float4*>(r + o)[qb];
        dd.x = fmaf(a4.x, pv.x, dd.x); dd.y = fmaf(a4.y, pv.y, dd.y);
        dd.z = fmaf(a4.z, pv.z, dd.z); dd.w = fmaf(a4.w, pv.w, dd.w);
        rv.x = fmaf(-a4.x, qv.x, rv.x); rv.y = fmaf(-a4.y, qv.y, rv.y);
        rv.z = fmaf(-a4.z, qv.z, rv.z); rv.w = fmaf(-a4.w, qv.w, rv.w);
        reinterpret_cast<float4*>(d + o)[qb] = dd;
        reinterpret_cast<float4*>(r + o)[qb] = rv;
        acc[0] += (double)(dv.x * rv.x * rv.x); acc[4] += (double)(rv.x * rv.x);
        acc[1] += (double)(dv.y * rv.y * rv.y); acc[5] += (double)(rv.y * rv.y);
        acc[2] += (double)(dv.z * rv.z * rv.z); acc[6] += (double)(rv.z * rv.z);
        acc[3] += (double)(dv.w * rv.w * rv.w); acc[7] += (double)(rv.w * rv.w);
      }
    }
    if (G == 1) {
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const size_t o = ((size_t)blockIdx.x * Rp + 4 * qb + u) * 2;
        partial[o] = acc[u];
        partial[o + 1] = acc[4 + u];
      }
    } else {
#pragma unroll
      for (int u = 0; u < 8; ++u) sh[((size_t)g * Q + qb) * 8 + u] = acc[u];
    }
  }
  if (G > 1) {
    __syncthreads();
    for (int qb = t; qb < Q; qb += 256) {
      double s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
      for (int gg = 0; gg < G; ++gg)
#pragma unroll
        for (int u = 0; u < 8; ++u) s[u] += sh[((size_t)gg * Q + qb) * 8 + u];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const size_t o = ((size_t)blockIdx.x * Rp + 4 * qb + u) * 2;
        partial[o] = s[u];
        partial[o + 1] = s[4 + u];
      }
    }
  }
}

struct Scal {
  float* alpha;   // [Rp]
  float* beta;    // [Rp]
  double* gamma;  // [Rp] (dinv r).r of the inner system
  double* rho0;   // [Rp] initial inner r.r
  double* res;    // [Rp] FP64 ||b - K x|| / ||b||
  double* bnorm;  // [Rp]
  int* act;       // [Rp] inner iteration active
  int* done;      // [Rp] converged (outer)
  int* its;       // [Rp] inner iterations (operator applications) in total
  int* its_step;  // [Rp] inner iterations in the current inner solve
  int* breakdown; // [Rp]
  int* n_active;  // [1]
};

// Per-realization sum of NV interleaved partials over n rows, 32 realizations x
// 32 row-groups per CTA; fixed summation order (row-group sequential, then the
// 32 groups in order), so results are reproducible and independent of the batch.
template <int NV>
__device__ __forceinline__ void reduce_rows(const double* __restrict__ partial, int n, int Rp, double (&out)[NV]) {
  __shared__ double sh[32][NV][33];
  const int lane = threadIdx.x & 31, g = threadIdx.x >> 5;
  const int r = blockIdx.x * 32 + lane;
  double acc[NV];
#pragma unroll
  for (int q = 0; q < NV; ++q) acc[q] = 0.0;
  for (int t = g; t < n; t += 32)
#pragma unroll
    for (int q = 0; q < NV; ++q) acc[q] += partial[((size_t)t * Rp + r) * NV + q];
#pragma unroll
  for (int q = 0; q < NV; ++q) sh[g][q][lane] = acc[q];
  __syncthreads();
#pragma unroll
  for (int q = 0; q < NV; ++q) {
    double s = 0.0;
    for (int gg = 0; gg < 32; ++gg) s += sh[gg][q][lane];
    out[q] = s;
  }
}

__global__ void __launch_bounds__(1024) k_alpha(int Rp, int n_tiles, const double* __restrict__ partial, Scal s) {
  double v[1];
  reduce_rows<1>(partial, n_tiles, Rp, v);
  if (threadIdx.x >= 32) return;
  const int r = blockIdx.x * 32 + threadIdx.x;
  const double pq = v[0];
  float a = 0.f;
  if (s.act[r]) {
    if (!(pq > 0.0)) {
      s.act[r] = 0; s.breakdown[r] = 1;
    } else {
      a = (float)(s.gamma[r] / pq);
      s.its[r] += 1;
      s.its_step[r] += 1;
    }
  }
  s.alpha[r] = a;
}

__global__ void __launch_bounds__(1024) k_beta(int Rp, int n_blk, const double* __restrict__ partial, Scal s,
                                               double eta2, int inner_max) {
  double v[2];
  reduce_rows<2>(partial, n_blk, Rp, v);
  const int r = blockIdx.x * 32 + threadIdx.x;
  int active = 0;
  if (threadIdx.x < 32) {
    const double g = v[0], rho = v[1];
    float b = 0.f;
    if (s.act[r]) {
      if (rho <= eta2 * s.rho0[r] || s.its_step[r] >= inner_max || !(rho == rho)) {
        s.act[r] = 0;
      } else {
        b = (float)(g / s.gamma[r]);
        s.gamma[r] = g;
        active = 1;
      }
    }
    s.beta[r] = b;
  }
  active = __syncthreads_count(active);
  if (threadIdx.x == 0 && active) atomicAdd(s.n_active, active);
}

__global__ void __launch_bounds__(1024) k_resid_scalars(int Rp, int n_tiles, const double* __restrict__ partial,
                                                        Scal s, double tol) {
  double v[2];
  reduce_rows<2>(partial, n_tiles, Rp, v);
  const int r = blockIdx.x * 32 + threadIdx.x;
  int active = 0;
  if (threadIdx.x < 32) {
    const double rr = v[0], g = v[1];
    const double bn = s.bnorm[r];
    const double rel = bn > 0 ? sqrt(rr) / bn : 0.0;
    s.res[r] = rel;
    if (!s.done[r] && (bn <= 1e-25 || rel < tol)) s.done[r] = 1;
    const int a = s.done[r] ? 0 : 1;
    s.act[r] = a;
    s.gamma[r] = g;
    s.rho0[r] = rr;
    s.beta[r] = 0.f;
    s.its_step[r] = 0;
    active = a;
  }
  active = __syncthreads_count(active);
  if (threadIdx.x == 0 && active) atomicAdd(s.n_active, active);
}

__global__ void k_lattice_rhs(int n_dofs, const int* __restrict__ free_rows, const double* __restrict__ b_dof,
                              double* __restrict__ b_lat) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n_dofs) b_lat[free_rows[i]] = b_dof[i];
}

// X[r][dof] = x[(row(dof))*Rp + r] through a 32x32 shared-memory transpose.
__global__ void k_gather_solution(int n_dofs, int R, int Rp, const int* __restrict__ free_rows,
                                  const double* __restrict__ x, double* __restrict__ X) {
  __shared__ double tile[32][33];
  const int d0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
  const int tx = threadIdx.x, ty = threadIdx.y;  // 32 x 8
  for (int q = ty; q < 32; q += 8) {
    const int d = d0 + q;
    tile[q][tx] = (d < n_dofs) ? x[(size_t)free_rows[d] * Rp + r0 + tx] : 0.0;
  }
  __syncthreads();
  for (int q = ty; q < 32; q += 8) {
    const int r = r0 + q, d = d0 + tx;
    if (r < R && d < n_dofs) X[(size_t)r * n_dofs + d] = tile[tx][q];
  }
}

__global__ void k_gather_tip(int R, int Rp, int row, const double* __restrict__ x, double* __restrict__ tip) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r < R) tip[r] = x[(size_t)row * Rp + r];
}

__global__ void k_set_bnorm(int R, int Rp, double bn, double* __restrict__ bnorm) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r < Rp) bnorm[r] = r < R ? bn : 0.0;
}

}  // namespace

int block_mixed_solve(Context* ctx, Mesh* m, double nu, const double* d_E64, const float* d_E32, int R, int Rp,
                      const double* d_b_dof, int max_it, double tol, int tip_dof, double* d_X, BatchOut out) {
  if (!m->structured) return set_error(ctx, MSG_ERR_NOT_STRUCTURED, "mesh is not a structured cube lattice");
  Lattice L;
  L.nx = m->nx; L.ny = m->ny; L.nz = m->nz;
  L.NX = m->nx + 1; L.NY = m->ny + 1; L.NZ = m->nz + 1;
  L.Rp = Rp;
  L.tiles_j = (L.NY + kTJ - 1) / kTJ;
  const int tiles_k = (L.NZ + kTK - 1) / kTK;
  const int n_tiles = L.tiles_j * tiles_k;
  const int nn = m->n_nodes;
  const size_t nvec = (size_t)nn * 3 * Rp;

  double K576[576];
  MSG_TRY(unit_cube_khat(ctx, m->h, nu, K576));
  KhatF KF;
  KhatD KD;
  for (int i = 0; i < 576; ++i) { KD.k[i] = K576[i]; KF.k[i] = (float)K576[i]; }
  const double kdiag = K576[0];

  DevMem x0, x1, r32, p0, p1, q, d, dinv, blat, part_op, part_up, scal;
  MSG_TRY(x0.alloc(ctx, sizeof(double) * nvec));
  MSG_TRY(x1.alloc(ctx, sizeof(double) * nvec));
  MSG_TRY(r32.alloc(ctx, sizeof(float) * nvec));
  MSG_TRY(p0.alloc(ctx, sizeof(float) * nvec));
  MSG_TRY(p1.alloc(ctx, sizeof(float) * nvec));
  MSG_TRY(q.alloc(ctx, sizeof(float) * nvec));
  MSG_TRY(d.alloc(ctx, sizeof(float) * nvec));
  MSG_TRY(dinv.alloc(ctx, sizeof(float) * (size_t)nn * Rp));
  MSG_TRY(blat.alloc(ctx, sizeof(double) * (size_t)nn * 3));
  const int n_upd = std::min(nn, ctx->sm_count * 4);
  MSG_TRY(part_op.alloc(ctx, sizeof(double) * (size_t)n_tiles * Rp * 2));
  MSG_TRY(part_up.alloc(ctx, sizeof(double) * (size_t)n_upd * Rp * 2));
  const size_t scal_bytes = (sizeof(float) * 2 + sizeof(double) * 4 + sizeof(int) * 5) * (size_t)Rp + 64;
  MSG_TRY(scal.alloc(ctx, scal_bytes));
  cudaStream_t st = ctx->stream;
  MSG_CUDA(ctx, cudaMemsetAsync(scal.ptr, 0, scal_bytes, st));
  Scal s;
  {
    char* base = scal.as<char>();
    s.alpha = (float*)base; base += sizeof(float) * Rp;
    s.beta = (float*)base; base += sizeof(float) * Rp;
    s.gamma = (double*)base; base += sizeof(double) * Rp;
    s.rho0 = (double*)base; base += sizeof(double) * Rp;
    s.res = (double*)base; base += sizeof(double) * Rp;
    s.bnorm = (double*)base; base += sizeof(double) * Rp;
    s.act = (int*)base; base += sizeof(int) * Rp;
    s.done = (int*)base; base += sizeof(int) * Rp;
    s.its = (int*)base; base += sizeof(int) * Rp;
    s.its_step = (int*)base; base += sizeof(int) * Rp;
    s.breakdown = (int*)base; base += sizeof(int) * Rp;
    s.n_active = (int*)base;
  }
  // b in lattice layout and ||b|| (one load vector for the whole batch)
  MSG_CUDA(ctx, cudaMemsetAsync(blat.ptr, 0, sizeof(double) * (size_t)nn * 3, st));
  k_lattice_rhs<<<(m->n_dofs + 255) / 256, 256, 0, st>>>(m->n_dofs, m->d_free_rows.as<int>(), d_b_dof,
                                                         blat.as<double>());
  std::vector<double> hb(m->n_dofs);
  MSG_CUDA(ctx, cudaMemcpyAsync(hb.data(), d_b_dof, sizeof(double) * m->n_dofs, cudaMemcpyDeviceToHost, st));
  MSG_CUDA(ctx, cudaStreamSynchronize(st));
  double bb = 0;
  for (double v : hb) bb += v * v;
  k_set_bnorm<<<(Rp + 127) / 128, 128, 0, st>>>(R, Rp, std::sqrt(bb), s.bnorm);
  MSG_CUDA(ctx, cudaMemsetAsync(x0.ptr, 0, sizeof(double) * nvec, st));
  MSG_CUDA(ctx, cudaMemsetAsync(d.ptr, 0, sizeof(float) * nvec, st));
  MSG_CUDA(ctx, cudaMemsetAsync(p0.ptr, 0, sizeof(float) * nvec, st));
  MSG_CUDA(ctx, cudaMemsetAsync(p1.ptr, 0, sizeof(float) * nvec, st));
  k_dinv<<<nn, 128, 0, st>>>(L, kdiag, d_E32, dinv.as<float>());
  count_launch(ctx, 3);
  MSG_CUDA(ctx, cudaGetLastError());

  const dim3 op_grid(n_tiles, Rp / 32), op_block(32, kWarps);
  const int Q = Rp / 4;
  const int G = Q >= 256 ? 1 : 256 / Q;
  const size_t upd_smem = G > 1 ? sizeof(double) * (size_t)G * Q * 8 : 0;
  const int sblocks = Rp / 32;  // scalar kernels: 32 realizations x 32 row groups per CTA

  cudaEvent_t ev[8];  // 0-3 host-side phases, 4-7 captured around the first operator / update launch
  for (auto& e : ev) MSG_CUDA(ctx, cudaEventCreate(&e));
  float t_resid = 0.f, t_inner = 0.f;

  const int chunk = std::max(2, ctx->chunk & ~1);
  cudaGraphExec_t gexec = nullptr;
  {
    cudaGraph_t g;
    MSG_CUDA(ctx, cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    for (int it = 0; it < chunk; ++it) {
      float* pold = (it & 1) ? p1.as<float>() : p0.as<float>();
      float* pnew = (it & 1) ? p0.as<float>() : p1.as<float>();
      // cudaEventRecordExternal: a real event-record node in the graph (plain
      // records during capture only order streams)
      if (it == 0) cudaEventRecordWithFlags(ev[4], st, cudaEventRecordExternal);
      k_inner_op<<<op_grid, op_block, 0, st>>>(L, KF, r32.as<float>(), pold, pnew, dinv.as<float>(), d_E32,
                                               m->d_mask.as<uint8_t>(), s.beta, q.as<float>(), part_op.as<double>());
      if (it == 0) cudaEventRecordWithFlags(ev[5], st, cudaEventRecordExternal);
      k_alpha<<<sblocks, 1024, 0, st>>>(Rp, n_tiles, part_op.as<double>(), s);
      if (it == 0) cudaEventRecordWithFlags(ev[6], st, cudaEventRecordExternal);
      k_update<<<n_upd, 256, upd_smem, st>>>(nn, Rp, s.alpha, pnew, q.as<float>(), d.as<float>(), r32.as<float>(),
                                             dinv.as<float>(), part_up.as<double>());
      if (it == 0) cudaEventRecordWithFlags(ev[7], st, cudaEventRecordExternal);
      cudaMemsetAsync(s.n_active, 0, sizeof(int), st);
      k_beta<<<sblocks, 1024, 0, st>>>(Rp, n_upd, part_up.as<double>(), s, ctx->inner_tol * ctx->inner_tol, ctx->inner_max);
    }
    cudaError_t e = cudaStreamEndCapture(st, &g);
    if (e != cudaSuccess) return cuda_error(ctx, e, "capture inner chunk");
    e = cudaGraphInstantiate(&gexec, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return cuda_error(ctx, e, "instantiate inner chunk");
  }

  int* h_active = nullptr;
  MSG_CUDA(ctx, cudaMallocHost(&h_active, sizeof(int)));
  int status = MSG_OK;
  int total_inner = 0;
  DevMem* xc = &x0;
  DevMem* xn = &x1;
  for (int outer = 0; outer < 1000; ++outer) {
    MSG_CUDA(ctx, cudaMemsetAsync(s.n_active, 0, sizeof(int), st));
    cudaEventRecord(ev[0], st);
    k_resid_op<<<op_grid, op_block, 0, st>>>(L, KD, xc->as<double>(), d.as<float>(), xn->as<double>(),
                                             blat.as<double>(), d_E64, m->d_mask.as<uint8_t>(), dinv.as<float>(),
                                             r32.as<float>(), part_op.as<double>());
    k_resid_scalars<<<sblocks, 1024, 0, st>>>(Rp, n_tiles, part_op.as<double>(), s, tol);
    cudaEventRecord(ev[1], st);
    count_launch(ctx, 2);
    std::swap(xc, xn);
    MSG_CUDA(ctx, cudaMemcpyAsync(h_active, s.n_active, sizeof(int), cudaMemcpyDeviceToHost, st));
    MSG_CUDA(ctx, cudaStreamSynchronize(st));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ev[0], ev[1]);
    t_resid += ms;
    if (*h_active == 0) break;
    if (total_inner >= max_it) { status = MSG_ERR_NOT_CONVERGED; break; }
    MSG_CUDA(ctx, cudaMemsetAsync(d.ptr, 0, sizeof(float) * nvec, st));
    cudaEventRecord(ev[2], st);
    while (true) {
      cudaError_t e = cudaGraphLaunch(gexec, st);
      if (e != cudaSuccess) { cudaFreeHost(h_active); cudaGraphExecDestroy(gexec); return cuda_error(ctx, e, "inner chunk"); }
      count_launch(ctx, 4 * chunk);
      total_inner += chunk;
      MSG_CUDA(ctx, cudaMemcpyAsync(h_active, s.n_active, sizeof(int), cudaMemcpyDeviceToHost, st));
      MSG_CUDA(ctx, cudaStreamSynchronize(st));
      float op_ms = 0.f, up_ms = 0.f;
      if (cudaEventElapsedTime(&op_ms, ev[4], ev[5]) == cudaSuccess &&
          cudaEventElapsedTime(&up_ms, ev[6], ev[7]) == cudaSuccess) {
        ctx->op_ms_sum += op_ms;
        ctx->upd_ms_sum += up_ms;
        ctx->op_samples += 1;
      }
      cudaGetLastError();
      if (*h_active == 0 || total_inner >= max_it) break;
    }
    cudaEventRecord(ev[3], st);
    MSG_CUDA(ctx, cudaStreamSynchronize(st));
    cudaEventElapsedTime(&ms, ev[2], ev[3]);
    t_inner += ms;
  }
  cudaFreeHost(h_active);
  cudaGraphExecDestroy(gexec);
  for (auto& e : ev) cudaEventDestroy(e);
  ctx->t_phase[1] = t_inner;
  ctx->t_phase[3] = t_resid;

  // outputs
  if (d_X) {
    dim3 g((m->n_dofs + 31) / 32, Rp / 32);
    k_gather_solution<<<g, dim3(32, 8), 0, st>>>(m->n_dofs, R, Rp, m->d_free_rows.as<int>(), xc->as<double>(), d_X);
    count_launch(ctx);
  }
  DevMem tipbuf;
  if (out.tip && tip_dof >= 0 && tip_dof < m->n_dofs) {
    int row = 0;
    MSG_CUDA(ctx, cudaMemcpyAsync(&row, m->d_free_rows.as<int>() + tip_dof, sizeof(int), cudaMemcpyDeviceToHost, st));
    MSG_CUDA(ctx, cudaStreamSynchronize(st));
    MSG_TRY(tipbuf.alloc(ctx, sizeof(double) * Rp));
    k_gather_tip<<<(R + 127) / 128, 128, 0, st>>>(R, Rp, row, xc->as<double>(), tipbuf.as<double>());
    count_launch(ctx);
    MSG_CUDA(ctx, cudaMemcpyAsync(out.tip, tipbuf.ptr, sizeof(double) * R, cudaMemcpyDeviceToHost, st));
  }
  std::vector<int> its(Rp), brk(Rp), done(Rp);
  std::vector<double> res(Rp);
  MSG_CUDA(ctx, cudaMemcpyAsync(its.data(), s.its, sizeof(int) * Rp, cudaMemcpyDeviceToHost, st));
  MSG_CUDA(ctx, cudaMemcpyAsync(brk.data(), s.breakdown, sizeof(int) * Rp, cudaMemcpyDeviceToHost, st));
  MSG_CUDA(ctx, cudaMemcpyAsync(done.data(), s.done, sizeof(int) * Rp, cudaMemcpyDeviceToHost, st));
  MSG_CUDA(ctx, cudaMemcpyAsync(res.data(), s.res, sizeof(double) * Rp, cudaMemcpyDeviceToHost, st));
  MSG_CUDA(ctx, cudaStreamSynchronize(st));
  MSG_CUDA(ctx, cudaGetLastError());
  for (int r = 0; r < R; ++r) {
    if (out.iterations) out.iterations[r] = its[r];
    if (out.rel_res) out.rel_res[r] = res[r];
    if (!done[r] && status == MSG_OK) status = brk[r] ? MSG_ERR_BREAKDOWN : MSG_ERR_NOT_CONVERGED;
  }
  if (status != MSG_OK)
    return set_error(ctx, status, "mixed batched solve: %s", status == MSG_ERR_BREAKDOWN ? "PCG breakdown" : "not converged");
  return MSG_OK;
}

}  // namespace msg
