// Batched mixed-precision Monte Carlo solve on any Hexa8 mesh (distorted or
// unstructured): the path of MonteCarloAnalyzerWithStochasticMaterial.SolveNormal
// (ISAAR.MSolve.Analyzers/MonteCarloAnalyzerWithStochasticMaterial.cs:232-296)
// for all realizations at once, where the cube-lattice operators do not apply.
//
// The stiffness of element e in realization r is K_e = E_{e,r} Khat_e with
// Khat_e the element's stiffness at E = 1 (the constitutive matrix is linear in
// E; Hexa8WithStochasticMaterial.cs:61-110 evaluates E once per element), so
// Khat_e is computed once per mesh and shared by every realization. The
// operator is applied node by node: the rows of node n are
//   y_n = sum over the elements e around n (corner a of e) of
//         E_{e,r} Khat_e[3a .. 3a+2][0 .. 23] u_e,
// one warp per node and 32 realizations (realization innermost, every vector
// access one 128-byte line), the 72 values of the corner's rows read as
// broadcast loads. Each output is written once and the sum over the elements
// runs in a fixed order: no atomics, results deterministic and independent of
// the batch.
//
// Loop: Jacobi-preconditioned CG per realization with FP32 vectors and the
// FP32 operator, the iterate x in FP64 through an FP32 correction d (x += d at
// every true residual), and reliable updates: when a realization's recursive
// ||r|| has dropped by `reliable_delta` since its last true residual, or below
// tol ||b|| / 2, or it reached the iteration limit, r = b - K x is formed with
// the FP64 operator for every running realization;
// a realization whose FP64 true relative residual is below tol stops, the
// others continue from the true residual with their search directions kept
// (residual replacement). Per-realization sums go through [block][Rp] partial
// arrays added in block order.
#include <algorithm>
#include <vector>

#include "msg_internal.h"

namespace msg {
namespace {

constexpr int kEbeWarps = 8;  // warps (nodes in flight) per CTA
constexpr int kEbeCheck = 8;  // iterations between host reads of the loop flags

// Khat_e in the per-corner layout (FP64 and FP32): entry [e][a][b][c2][r] =
// Khat_e[3a + r][3b + c2], i.e. the 72 values the rows of corner a need, with
// the three row components innermost.
__global__ void k_ebe_unpack(int ne, const double* __restrict__ K300, double* __restrict__ K64,
                             float* __restrict__ K32) {
  const int e = blockIdx.x;
  if (e >= ne) return;
  for (int i = threadIdx.x; i < 576; i += blockDim.x) {
    const int a = i / 72, rem = i % 72, b = rem / 9, c2 = (rem % 9) / 3, r = rem % 3;
    const double v = K300[(size_t)e * 300 + packed_index(3 * a + r, 3 * b + c2)];
    K64[(size_t)e * 576 + i] = v;
    K32[(size_t)e * 576 + i] = (float)v;
  }
}

// CTA sum (fixed warp order) of the lanes' values into partial[blockIdx.x][Rp]
// at realizations col0 .. col0 + 31 (default: this CTA's realization group).
__device__ __forceinline__ void ebe_block_partial(double v, double* sh, double* __restrict__ partial, int Rp,
                                                  int col0 = -1) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  sh[w * 32 + lane] = v;
  __syncthreads();
  if (w == 0) {
    double s = 0.0;
    for (int i = 0; i < kEbeWarps; ++i) s += sh[i * 32 + lane];
    partial[(size_t)blockIdx.x * Rp + (col0 < 0 ? blockIdx.y * 32 : col0) + lane] = s;
  }
  __syncthreads();
}

// Node rows of K u in FP32 for G realization groups of 32 (realizations
// rb + 32 g + lane): the corner's 72 values as 18 float4 broadcast loads (each
// per-corner block starts on a 288-byte boundary), used by all G groups. A
// broadcast load fills 32 lanes' registers, so its cost in the load
// writeback path is shared by the G groups; every realization's arithmetic
// (order of the products and sums) is the same for every G.
template <int G>
__device__ __forceinline__ void ebe_rows32(int n, int Rp, int rb, const int* __restrict__ inc_ptr,
                                           const int* __restrict__ inc, const int* __restrict__ conn,
                                           const float* __restrict__ Kh, const float* __restrict__ E,
                                           const float* __restrict__ u, float (&y)[G][3]) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int g = 0; g < G; ++g) y[g][0] = y[g][1] = y[g][2] = 0.f;
  const int k1 = __ldg(inc_ptr + n + 1);
  for (int k = __ldg(inc_ptr + n); k < k1; ++k) {
    const int ea = __ldg(inc + k);
    const int e = ea >> 3, a = ea & 7;
    const float4* __restrict__ K4 = reinterpret_cast<const float4*>(Kh + (size_t)e * 576 + 72 * a);
    const int4 c0 = __ldg(reinterpret_cast<const int4*>(conn) + 2 * (size_t)e);
    const int4 c1 = __ldg(reinterpret_cast<const int4*>(conn) + 2 * (size_t)e + 1);
    const int nb[8] = {c0.x, c0.y, c0.z, c0.w, c1.x, c1.y, c1.z, c1.w};
    float t[G][3];
#pragma unroll
    for (int g = 0; g < G; ++g) t[g][0] = t[g][1] = t[g][2] = 0.f;
#pragma unroll
    for (int q = 0; q < 6; ++q) {  // 4 columns (3 float4, 12 values) per step
      float kv[12];
      *reinterpret_cast<float4*>(kv) = __ldg(K4 + 3 * q);
      *reinterpret_cast<float4*>(kv + 4) = __ldg(K4 + 3 * q + 1);
      *reinterpret_cast<float4*>(kv + 8) = __ldg(K4 + 3 * q + 2);
#pragma unroll
      for (int s = 0; s < 4; ++s) {
        const int j = 4 * q + s;  // column 3b + c2
        const float* __restrict__ ub = u + ((size_t)nb[j / 3] * 3 + j % 3) * Rp + rb + lane;
#pragma unroll
        for (int g = 0; g < G; ++g) {
          const float uv = ub[32 * g];
          t[g][0] = fmaf(kv[3 * s], uv, t[g][0]);
          t[g][1] = fmaf(kv[3 * s + 1], uv, t[g][1]);
          t[g][2] = fmaf(kv[3 * s + 2], uv, t[g][2]);
        }
      }
    }
#pragma unroll
    for (int g = 0; g < G; ++g) {
      const float Ee = E[(size_t)e * Rp + rb + 32 * g + lane];
      y[g][0] = fmaf(Ee, t[g][0], y[g][0]);
      y[g][1] = fmaf(Ee, t[g][1], y[g][1]);
      y[g][2] = fmaf(Ee, t[g][2], y[g][2]);
    }
  }
}

// The same rows in FP64 (true residuals).
__device__ __forceinline__ void ebe_rows64(int n, int Rp, int rr, const int* __restrict__ inc_ptr,
                                           const int* __restrict__ inc, const int* __restrict__ conn,
                                           const double* __restrict__ Kh, const double* __restrict__ E,
                                           const double* __restrict__ u, double (&y)[3]) {
  y[0] = y[1] = y[2] = 0.0;
  const int k1 = __ldg(inc_ptr + n + 1);
  for (int k = __ldg(inc_ptr + n); k < k1; ++k) {
    const int ea = __ldg(inc + k);
    const int e = ea >> 3, a = ea & 7;
    const double2* __restrict__ K2 = reinterpret_cast<const double2*>(Kh + (size_t)e * 576 + 72 * a);
    const int4 c0 = __ldg(reinterpret_cast<const int4*>(conn) + 2 * (size_t)e);
    const int4 c1 = __ldg(reinterpret_cast<const int4*>(conn) + 2 * (size_t)e + 1);
    const int nb[8] = {c0.x, c0.y, c0.z, c0.w, c1.x, c1.y, c1.z, c1.w};
    double t0 = 0.0, t1 = 0.0, t2 = 0.0;
#pragma unroll
    for (int q = 0; q < 12; ++q) {  // 2 columns (3 double2, 6 values) per step
      const double2 ka = __ldg(K2 + 3 * q), kb = __ldg(K2 + 3 * q + 1), kc = __ldg(K2 + 3 * q + 2);
      const int j0 = 2 * q, j1 = 2 * q + 1;
      const double u0 = u[((size_t)nb[j0 / 3] * 3 + j0 % 3) * Rp + rr];
      const double u1 = u[((size_t)nb[j1 / 3] * 3 + j1 % 3) * Rp + rr];
      t0 = fma(ka.x, u0, t0);
      t1 = fma(ka.y, u0, t1);
      t2 = fma(kb.x, u0, t2);
      t0 = fma(kb.y, u1, t0);
      t1 = fma(kc.x, u1, t1);
      t2 = fma(kc.y, u1, t2);
    }
    const double Ee = E[(size_t)e * Rp + rr];
    y[0] = fma(Ee, t0, y[0]);
    y[1] = fma(Ee, t1, y[1]);
    y[2] = fma(Ee, t2, y[2]);
  }
}

// q = K p (FP32, constrained components 0) and the partial p.q per realization;
// each CTA covers 32 G realizations (grid.y = Rp / (32 G)).
template <int G>
__global__ void __launch_bounds__(32 * kEbeWarps) k_ebe_apply32(int n_nodes, int Rp, const int* __restrict__ inc_ptr,
                                                               const int* __restrict__ inc,
                                                               const int* __restrict__ conn,
                                                               const float* __restrict__ Kh,
                                                               const float* __restrict__ E,
                                                               const uint8_t* __restrict__ mask,
                                                               const float* __restrict__ p, float* __restrict__ q,
                                                               double* __restrict__ partial) {
  __shared__ double sh[kEbeWarps * 32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int rb = blockIdx.y * 32 * G;
  double pq[G];
#pragma unroll
  for (int g = 0; g < G; ++g) pq[g] = 0.0;
  for (int n = blockIdx.x * kEbeWarps + w; n < n_nodes; n += gridDim.x * kEbeWarps) {
    float y[G][3];
    ebe_rows32<G>(n, Rp, rb, inc_ptr, inc, conn, Kh, E, p, y);
    const unsigned mk = __ldg(mask + n);
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int g = 0; g < G; ++g) {
        const size_t o = ((size_t)n * 3 + c) * Rp + rb + 32 * g + lane;
        const float v = ((mk >> c) & 1u) ? 0.f : y[g][c];
        q[o] = v;
        pq[g] += (double)p[o] * (double)v;
      }
  }
#pragma unroll
  for (int g = 0; g < G; ++g) ebe_block_partial(pq[g], sh, partial, Rp, rb + 32 * g);
}

// FP64 true residual r = b - K x (b one node-layout vector shared by every
// realization; constrained components 0) of the running realizations into the
// FP32 residual; partials ||r||^2 and (dinv r).r.
__global__ void __launch_bounds__(32 * kEbeWarps) k_ebe_resid64(int n_nodes, int Rp, const int* __restrict__ inc_ptr,
                                                               const int* __restrict__ inc,
                                                               const int* __restrict__ conn,
                                                               const double* __restrict__ Kh,
                                                               const double* __restrict__ E,
                                                               const uint8_t* __restrict__ mask,
                                                               const double* __restrict__ b,
                                                               const double* __restrict__ x,
                                                               const float* __restrict__ dinv,
                                                               const int* __restrict__ done,
                                                               float* __restrict__ r32, double* __restrict__ part_rr,
                                                               double* __restrict__ part_zr) {
  __shared__ double sh[kEbeWarps * 32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int rr = blockIdx.y * 32 + lane;
  const bool run = done[rr] == 0;
  double s_rr = 0.0, s_zr = 0.0;
  for (int n = blockIdx.x * kEbeWarps + w; n < n_nodes; n += gridDim.x * kEbeWarps) {
    double y[3];
    ebe_rows64(n, Rp, rr, inc_ptr, inc, conn, Kh, E, x, y);
    const unsigned mk = __ldg(mask + n);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const size_t o = ((size_t)n * 3 + c) * Rp + rr;
      const double v = ((mk >> c) & 1u) ? 0.0 : b[(size_t)n * 3 + c] - y[c];
      const float v32 = (float)v;
      if (run) r32[o] = v32;
      s_rr += v * v;
      s_zr += (double)(dinv[o] * v32) * (double)v32;
    }
  }
  ebe_block_partial(s_rr, sh, part_rr, Rp);
  ebe_block_partial(s_zr, sh, part_zr, Rp);
}

// Jacobi diagonal of every realization: dinv = 1 / sum_e E_{e,r} Khat_e[3a+c][3a+c]
// (1 on constrained components).
__global__ void k_ebe_dinv(int n_nodes, int Rp, const int* __restrict__ inc_ptr, const int* __restrict__ inc,
                           const double* __restrict__ Kh, const double* __restrict__ E,
                           const uint8_t* __restrict__ mask, float* __restrict__ dinv) {
  const int n = blockIdx.x;
  if (n >= n_nodes) return;
  for (int rr = threadIdx.x; rr < Rp; rr += blockDim.x) {
    double d[3] = {0.0, 0.0, 0.0};
    for (int k = inc_ptr[n]; k < inc_ptr[n + 1]; ++k) {
      const int e = inc[k] >> 3, a = inc[k] & 7;
      const double Ee = E[(size_t)e * Rp + rr];
#pragma unroll
      for (int c = 0; c < 3; ++c) d[c] += Ee * Kh[(size_t)e * 576 + 72 * a + 9 * a + 4 * c];
    }
    const unsigned mk = mask[n];
#pragma unroll
    for (int c = 0; c < 3; ++c)
      dinv[((size_t)n * 3 + c) * Rp + rr] = (((mk >> c) & 1u) || !(d[c] > 0.0)) ? 1.f : (float)(1.0 / d[c]);
  }
}

// Per-realization loop state.
struct EbeScal {
  double* gamma;   // [Rp] (dinv r).r of the current residual
  double* rr_ref;  // [Rp] ||r||^2 at the last true residual
  double* bnorm;   // [Rp]
  double* res;     // [Rp] last FP64 true relative residual
  float* alpha;    // [Rp]
  float* beta;     // [Rp]
  int* done;       // [Rp] 0 running, 1 converged (or padding), 2 breakdown, 3 iteration limit
  int* its;        // [Rp] FP32 operator products
  int* flags;      // [2] realizations asking for a true residual, realizations still running
};

// x = 0, d = 0, r = b, p = dinv b (every realization the same b)
__global__ void k_ebe_init(size_t n3, int Rp, const double* __restrict__ b, const float* __restrict__ dinv,
                           double* __restrict__ x, float* __restrict__ d, float* __restrict__ r,
                           float* __restrict__ p) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n3 * Rp; i += (size_t)gridDim.x * blockDim.x) {
    const float bv = (float)b[i / Rp];
    x[i] = 0.0;
    d[i] = 0.f;
    r[i] = bv;
    p[i] = dinv[i] * bv;
  }
}

// x += d, d = 0: the FP32 correction accumulated since the last true residual
// folded into the FP64 iterate
__global__ void k_ebe_fold(size_t nv, double* __restrict__ x, float* __restrict__ d) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < nv; i += (size_t)gridDim.x * blockDim.x) {
    x[i] += (double)d[i];
    d[i] = 0.f;
  }
}

// Partials of ||b||^2 and (dinv b).b per realization (the residual at x = 0).
__global__ void __launch_bounds__(32 * kEbeWarps) k_ebe_bnorm(int n_nodes, int Rp, const double* __restrict__ b,
                                                             const float* __restrict__ dinv,
                                                             double* __restrict__ part_rr,
                                                             double* __restrict__ part_zr) {
  __shared__ double sh[kEbeWarps * 32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int rr = blockIdx.y * 32 + lane;
  double s_rr = 0.0, s_zr = 0.0;
  for (int n = blockIdx.x * kEbeWarps + w; n < n_nodes; n += gridDim.x * kEbeWarps)
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const double v = b[(size_t)n * 3 + c];
      const float v32 = (float)v;
      s_rr += v * v;
      s_zr += (double)(dinv[((size_t)n * 3 + c) * Rp + rr] * v32) * (double)v32;
    }
  ebe_block_partial(s_rr, sh, part_rr, Rp);
  ebe_block_partial(s_zr, sh, part_zr, Rp);
}

// Sum over the block partials of realization r by one warp: lane l adds blocks
// l, l + 32, ... in order, then a butterfly over the lanes (every lane gets the
// same bits: each step adds the same two values on both lanes of a pair).
__device__ __forceinline__ double ebe_sum(const double* __restrict__ part, int n_blocks, int Rp, int r) {
  const int lane = threadIdx.x & 31;
  double s = 0.0;
  for (int i = lane; i < n_blocks; i += 32) s += part[(size_t)i * Rp + r];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  return s;
}

// realization of this warp in the scalar kernels (one warp per realization)
__device__ __forceinline__ int ebe_warp_realization() { return (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5); }

// Starting scalars; a zero right-hand side (and padding) is done at once with x = 0.
__global__ void k_ebe_start(int R, int Rp, int n_blocks, const double* __restrict__ part_rr,
                            const double* __restrict__ part_zr, EbeScal s) {
  const int r = ebe_warp_realization();
  if (r >= Rp) return;
  const double bb = ebe_sum(part_rr, n_blocks, Rp, r), zr = ebe_sum(part_zr, n_blocks, Rp, r);
  if ((threadIdx.x & 31) != 0) return;
  s.bnorm[r] = sqrt(bb);
  s.rr_ref[r] = bb;
  s.gamma[r] = zr;
  s.alpha[r] = 0.f;
  s.beta[r] = 0.f;
  s.its[r] = 0;
  s.res[r] = bb > 0.0 ? 1.0 : 0.0;
  s.done[r] = (r >= R || !(bb > 0.0)) ? 1 : 0;
}

// alpha = gamma / p.q (breakdown when p.q <= 0 or not finite)
__global__ void k_ebe_alpha(int Rp, int n_blocks, const double* __restrict__ part_pq, EbeScal s) {
  const int r = ebe_warp_realization();
  if (r >= Rp) return;
  if (s.done[r]) {
    if ((threadIdx.x & 31) == 0) s.alpha[r] = 0.f;
    return;
  }
  const double pq = ebe_sum(part_pq, n_blocks, Rp, r);
  if ((threadIdx.x & 31) != 0) return;
  s.its[r] += 1;
  if (!(pq > 0.0) || !isfinite(pq)) {
    s.done[r] = 2;
    s.alpha[r] = 0.f;
    return;
  }
  s.alpha[r] = (float)(s.gamma[r] / pq);
}

// d += alpha p (the FP32 correction of the FP64 iterate), r -= alpha q,
// partials (dinv r).r and r.r
__global__ void __launch_bounds__(32 * kEbeWarps) k_ebe_update(int n_nodes, int Rp, const float* __restrict__ alpha,
                                                              const float* __restrict__ p,
                                                              const float* __restrict__ q,
                                                              const float* __restrict__ dinv,
                                                              float* __restrict__ d, float* __restrict__ r,
                                                              double* __restrict__ part_zr,
                                                              double* __restrict__ part_rr) {
  __shared__ double sh[kEbeWarps * 32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int rr = blockIdx.y * 32 + lane;
  const float al = alpha[rr];
  double s_zr = 0.0, s_rr = 0.0;
  for (int n = blockIdx.x * kEbeWarps + w; n < n_nodes; n += gridDim.x * kEbeWarps)
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const size_t o = ((size_t)n * 3 + c) * Rp + rr;
      d[o] = fmaf(al, p[o], d[o]);
      const float rv = fmaf(-al, q[o], r[o]);
      r[o] = rv;
      s_zr += (double)(dinv[o] * rv) * (double)rv;
      s_rr += (double)rv * (double)rv;
    }
  ebe_block_partial(s_zr, sh, part_zr, Rp);
  ebe_block_partial(s_rr, sh, part_rr, Rp);
}

// beta = gamma_new / gamma; a realization asks for a true residual when its
// recursive ||r||^2 is below tol2 ||b||^2 or delta2 times the last true one, or
// it reached the iteration limit.
__global__ void k_ebe_beta(int Rp, int n_blocks, const double* __restrict__ part_zr,
                           const double* __restrict__ part_rr, EbeScal s, double tol2, double delta2, int max_it) {
  const int r = ebe_warp_realization();
  if (r >= Rp) return;
  if (s.done[r]) {
    if ((threadIdx.x & 31) == 0) s.beta[r] = 0.f;
    return;
  }
  const double zr = ebe_sum(part_zr, n_blocks, Rp, r), rr = ebe_sum(part_rr, n_blocks, Rp, r);
  if ((threadIdx.x & 31) != 0) return;
  s.beta[r] = s.gamma[r] > 0.0 ? (float)(zr / s.gamma[r]) : 0.f;
  s.gamma[r] = zr;
  const double b2 = s.bnorm[r] * s.bnorm[r];
  if (rr < tol2 * b2 || rr < delta2 * s.rr_ref[r] || s.its[r] >= max_it) atomicAdd(s.flags, 1);
}

// After the FP64 true residual: converged realizations stop; the others keep
// their direction and continue from the true residual. flags[1] counts the
// realizations still running.
__global__ void k_ebe_true(int Rp, int n_blocks, const double* __restrict__ part_rr,
                           const double* __restrict__ part_zr, EbeScal s, double tol, int max_it) {
  const int r = ebe_warp_realization();
  if (r >= Rp) return;
  if (s.done[r]) return;
  const double rr = ebe_sum(part_rr, n_blocks, Rp, r), zr = ebe_sum(part_zr, n_blocks, Rp, r);
  if ((threadIdx.x & 31) != 0) return;
  const double err = s.bnorm[r] > 0.0 ? sqrt(rr) / s.bnorm[r] : 0.0;
  s.res[r] = err;
  s.rr_ref[r] = rr;
  s.gamma[r] = zr;
  if (err < tol) {
    s.done[r] = 1;
  } else if (s.its[r] >= max_it || !isfinite(err)) {
    s.done[r] = 3;
  } else {
    atomicAdd(s.flags + 1, 1);
  }
}

// p = dinv r + beta p
__global__ void k_ebe_dir(size_t n3, int Rp, const float* __restrict__ beta, const float* __restrict__ dinv,
                          const float* __restrict__ r, float* __restrict__ p) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n3 * Rp; i += (size_t)gridDim.x * blockDim.x)
    p[i] = fmaf(beta[i % Rp], p[i], dinv[i] * r[i]);
}

// X[r][dof] = x[free_rows[dof] * Rp + r] for the first R realizations
__global__ void k_ebe_gather(int n_dofs, int R, int Rp, const int* __restrict__ rows, const double* __restrict__ x,
                             double* __restrict__ X) {
  __shared__ double tile[32][33];
  const int d0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
  const int tx = threadIdx.x, ty = threadIdx.y;  // 32 x 8
  for (int q = ty; q < 32; q += 8) {
    const int d = d0 + q;
    tile[q][tx] = (d < n_dofs) ? x[(size_t)rows[d] * Rp + r0 + tx] : 0.0;
  }
  __syncthreads();
  for (int q = ty; q < 32; q += 8) {
    const int r = r0 + q, d = d0 + tx;
    if (r < R && d < n_dofs) X[(size_t)r * n_dofs + d] = tile[tx][q];
  }
}

__global__ void k_ebe_tip(int R, int Rp, int row, const double* __restrict__ x, double* __restrict__ tip) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r < R) tip[r] = x[(size_t)row * Rp + r];
}

}  // namespace

// Node -> (element, corner) incidence of a mesh: CSR over nodes, entries
// (e << 3 | a) in ascending element order (the fixed summation order).
static void ebe_incidence(const Mesh* m, std::vector<int>& ptr, std::vector<int>& inc) {
  ptr.assign(m->n_nodes + 1, 0);
  for (int e = 0; e < m->n_elems; ++e)
    for (int a = 0; a < 8; ++a) ++ptr[m->conn[8 * (size_t)e + a] + 1];
  for (int n = 0; n < m->n_nodes; ++n) ptr[n + 1] += ptr[n];
  inc.assign(std::max(1, ptr[m->n_nodes]), 0);
  std::vector<int> fill(ptr.begin(), ptr.end() - 1);
  for (int e = 0; e < m->n_elems; ++e)
    for (int a = 0; a < 8; ++a) inc[fill[m->conn[8 * (size_t)e + a]]++] = (e << 3) | a;
}

int ebe_mixed_solve(Context* ctx, Mesh* m, double nu, const KLDevice* kd, const double* d_xi, int R,
                    const double* d_b_dof, int max_it, double tol, int tip_dof, double* d_X, BatchOut out) {
  NvtxRange range("msg: batched element-by-element solve");
  if ((int64_t)m->n_elems * 8 >= ((int64_t)1 << 31) || m->n_nodes <= 0 || m->n_elems <= 0)
    return set_error(ctx, MSG_ERR_INVALID_ARGUMENT, "element-by-element batch: mesh size out of range");
  const int Rp = (R + 31) / 32 * 32;
  const int nn = m->n_nodes, ne = m->n_elems;
  const size_t n3 = 3 * (size_t)nn, nv = n3 * Rp;
  cudaStream_t st = ctx->stream;
  // per-mesh data: Khat_e in the per-corner layout (FP64, FP32), incidence
  std::vector<int> ptr, inc;
  ebe_incidence(m, ptr, inc);
  DevMem d_ptr, d_inc, d_K300, d_K64, d_K32, d_st;
  MSG_TRY(d_ptr.alloc(ctx, sizeof(int) * ptr.size()));
  MSG_TRY(d_inc.alloc(ctx, sizeof(int) * inc.size()));
  MSG_CUDA(ctx, cudaMemcpyAsync(d_ptr.ptr, ptr.data(), sizeof(int) * ptr.size(), cudaMemcpyHostToDevice, st));
  MSG_CUDA(ctx, cudaMemcpyAsync(d_inc.ptr, inc.data(), sizeof(int) * inc.size(), cudaMemcpyHostToDevice, st));
  MSG_TRY(d_K300.alloc(ctx, sizeof(double) * 300 * (size_t)ne));
  MSG_TRY(d_K64.alloc(ctx, sizeof(double) * 576 * (size_t)ne));
  MSG_TRY(d_K32.alloc(ctx, sizeof(float) * 576 * (size_t)ne));
  MSG_TRY(d_st.alloc(ctx, sizeof(int)));
  MSG_CUDA(ctx, cudaMemsetAsync(d_st.ptr, 0, sizeof(int), st));
  MSG_TRY(launch_h8_ke(ctx, ne, m->d_exyz.as<double>(), nullptr, 1.0, nu, d_K300.as<double>(), d_st.as<int>()));
  k_ebe_unpack<<<ne, 128, 0, st>>>(ne, d_K300.as<double>(), d_K64.as<double>(), d_K32.as<float>());
  count_launch(ctx);
  int neg = 0;
  MSG_CUDA(ctx, cudaMemcpyAsync(&neg, d_st.ptr, sizeof(int), cudaMemcpyDeviceToHost, st));
  MSG_CUDA(ctx, cudaStreamSynchronize(st));
  if (neg) return set_error(ctx, MSG_ERR_NEG_DET, "element with a non-positive Jacobian determinant");
  d_K300.release();
  // E of every element and realization [e][Rp]
  DevMem d_E64, d_E32;
  MSG_TRY(d_E64.alloc(ctx, sizeof(double) * (size_t)ne * Rp));
  MSG_TRY(d_E32.alloc(ctx, sizeof(float) * (size_t)ne * Rp));
  MSG_TRY(launch_kl_field(ctx, m, kd, R, Rp, d_xi, d_E64.as<double>(), d_E32.as<float>(), nullptr));
  // vectors [node*3 + c][Rp] and scalars
  DevMem d_x, d_d, d_r, d_p, d_q, d_dinv, d_bn, d_scal, d_part;
  MSG_TRY(d_x.alloc(ctx, sizeof(double) * nv));
  MSG_TRY(d_d.alloc(ctx, sizeof(float) * nv));
  MSG_TRY(d_r.alloc(ctx, sizeof(float) * nv));
  MSG_TRY(d_p.alloc(ctx, sizeof(float) * nv));
  MSG_TRY(d_q.alloc(ctx, sizeof(float) * nv));
  MSG_TRY(d_dinv.alloc(ctx, sizeof(float) * nv));
  MSG_TRY(d_bn.alloc(ctx, sizeof(double) * n3));
  MSG_CUDA(ctx, cudaMemsetAsync(d_bn.ptr, 0, sizeof(double) * n3, st));
  MSG_TRY(launch_dof_to_node(ctx, m, d_b_dof, d_bn.as<double>(), 1, 0, 0));
  const int gx = std::max(1, std::min((nn + kEbeWarps - 1) / kEbeWarps, ctx->sm_count * 4));
  const dim3 grid(gx, Rp / 32);
  MSG_TRY(d_scal.alloc(ctx, (sizeof(double) * 4 + sizeof(float) * 2 + sizeof(int) * 2) * (size_t)Rp + 64));
  EbeScal s;
  s.gamma = d_scal.as<double>();
  s.rr_ref = s.gamma + Rp;
  s.bnorm = s.rr_ref + Rp;
  s.res = s.bnorm + Rp;
  s.alpha = reinterpret_cast<float*>(s.res + Rp);
  s.beta = s.alpha + Rp;
  s.done = reinterpret_cast<int*>(s.beta + Rp);
  s.its = s.done + Rp;
  s.flags = s.its + Rp;
  MSG_TRY(d_part.alloc(ctx, sizeof(double) * 2 * (size_t)gx * Rp));  // two [gx][Rp] partial arrays
  double* part_a = d_part.as<double>();
  double* part_b = part_a + (size_t)gx * Rp;
  const int* dptr = d_ptr.as<int>();
  const int* dinc = d_inc.as<int>();
  const int* conn = m->d_conn.as<int>();
  const uint8_t* mask = m->d_mask.as<uint8_t>();
  const int sb = Rp / 8;  // scalar kernels: one warp per realization, 8 per CTA
  // realization groups of 32 per CTA of the FP32 operator: the largest of 8, 4,
  // 2, 1 that divides the group count (or the element_groups option when it does)
  const int ng = Rp / 32;
  int G = ng % 8 == 0 ? 8 : ng % 4 == 0 ? 4 : ng % 2 == 0 ? 2 : 1;
  if (ctx->element_groups > 0 && ng % ctx->element_groups == 0) G = ctx->element_groups;
  const dim3 grid_op(gx, ng / G);
  auto apply32 = [&]() {
    const float* K32 = d_K32.as<float>();
    const float* E32 = d_E32.as<float>();
    switch (G) {
      case 8:
        k_ebe_apply32<8><<<grid_op, 32 * kEbeWarps, 0, st>>>(nn, Rp, dptr, dinc, conn, K32, E32, mask,
                                                              d_p.as<float>(), d_q.as<float>(), part_a);
        break;
      case 4:
        k_ebe_apply32<4><<<grid_op, 32 * kEbeWarps, 0, st>>>(nn, Rp, dptr, dinc, conn, K32, E32, mask,
                                                              d_p.as<float>(), d_q.as<float>(), part_a);
        break;
      case 2:
        k_ebe_apply32<2><<<grid_op, 32 * kEbeWarps, 0, st>>>(nn, Rp, dptr, dinc, conn, K32, E32, mask,
                                                              d_p.as<float>(), d_q.as<float>(), part_a);
        break;
      default:
        k_ebe_apply32<1><<<grid_op, 32 * kEbeWarps, 0, st>>>(nn, Rp, dptr, dinc, conn, K32, E32, mask,
                                                              d_p.as<float>(), d_q.as<float>(), part_a);
    }
  };
  const int gv = (int)std::min<size_t>((nv + 255) / 256, (size_t)ctx->sm_count * 16);
  k_ebe_dinv<<<nn, 128, 0, st>>>(nn, Rp, dptr, dinc, d_K64.as<double>(), d_E64.as<double>(), mask,
                                 d_dinv.as<float>());
  k_ebe_init<<<gv, 256, 0, st>>>(n3, Rp, d_bn.as<double>(), d_dinv.as<float>(), d_x.as<double>(), d_d.as<float>(),
                                 d_r.as<float>(), d_p.as<float>());
  k_ebe_bnorm<<<grid, 32 * kEbeWarps, 0, st>>>(nn, Rp, d_bn.as<double>(), d_dinv.as<float>(), part_a, part_b);
  k_ebe_start<<<sb, 256, 0, st>>>(R, Rp, gx, part_a, part_b, s);
  count_launch(ctx, 4);
  MSG_CUDA(ctx, cudaGetLastError());
  const double delta2 = ctx->reliable_delta * ctx->reliable_delta, tol2 = 0.25 * tol * tol;
  int* h = ctx->h_flags;
  // every chunk adds kEbeCheck products to each running realization and a
  // realization at the limit forces a true residual, which stops it: the loop
  // ends after at most max_it / kEbeCheck + 1 chunks
  const int max_chunks = max_it / kEbeCheck + 2;
  for (int chunk = 0; chunk < max_chunks; ++chunk) {
    MSG_CUDA(ctx, cudaMemsetAsync(s.flags, 0, 2 * sizeof(int), st));
    for (int k = 0; k < kEbeCheck; ++k) {
      apply32();
      k_ebe_alpha<<<sb, 256, 0, st>>>(Rp, gx, part_a, s);
      k_ebe_update<<<grid, 32 * kEbeWarps, 0, st>>>(nn, Rp, s.alpha, d_p.as<float>(), d_q.as<float>(),
                                                     d_dinv.as<float>(), d_d.as<float>(), d_r.as<float>(), part_a,
                                                     part_b);
      k_ebe_beta<<<sb, 256, 0, st>>>(Rp, gx, part_a, part_b, s, tol2, delta2, max_it);
      k_ebe_dir<<<gv, 256, 0, st>>>(n3, Rp, s.beta, d_dinv.as<float>(), d_r.as<float>(), d_p.as<float>());
      count_launch(ctx, 5);
    }
    MSG_CUDA(ctx, cudaGetLastError());
    MSG_CUDA(ctx, cudaMemcpyAsync(h, s.flags, sizeof(int), cudaMemcpyDeviceToHost, st));
    MSG_CUDA(ctx, cudaStreamSynchronize(st));
    if (h[0] == 0) continue;
    // FP64 true residual of the running realizations, then stop or continue each
    k_ebe_fold<<<gv, 256, 0, st>>>(nv, d_x.as<double>(), d_d.as<float>());
    k_ebe_resid64<<<grid, 32 * kEbeWarps, 0, st>>>(nn, Rp, dptr, dinc, conn, d_K64.as<double>(), d_E64.as<double>(),
                                                    mask, d_bn.as<double>(), d_x.as<double>(), d_dinv.as<float>(),
                                                    s.done, d_r.as<float>(), part_a, part_b);
    k_ebe_true<<<sb, 256, 0, st>>>(Rp, gx, part_a, part_b, s, tol, max_it);
    count_launch(ctx, 3);
    MSG_CUDA(ctx, cudaGetLastError());
    MSG_CUDA(ctx, cudaMemcpyAsync(h + 1, s.flags + 1, sizeof(int), cudaMemcpyDeviceToHost, st));
    MSG_CUDA(ctx, cudaStreamSynchronize(st));
    if (h[1] == 0) break;
  }
  // results (a realization stops right after a fold, so d holds no correction
  // here unless the chunk bound ended the loop)
  k_ebe_fold<<<gv, 256, 0, st>>>(nv, d_x.as<double>(), d_d.as<float>());
  count_launch(ctx);
  if (d_X && m->n_dofs > 0) {
    const dim3 g((m->n_dofs + 31) / 32, Rp / 32);
    k_ebe_gather<<<g, dim3(32, 8), 0, st>>>(m->n_dofs, R, Rp, m->d_free_rows.as<int>(), d_x.as<double>(), d_X);
    count_launch(ctx);
  }
  if (out.tip && tip_dof >= 0 && tip_dof < m->n_dofs) {
    int row = 0;
    MSG_CUDA(ctx, cudaMemcpyAsync(&row, m->d_free_rows.as<int>() + tip_dof, sizeof(int), cudaMemcpyDeviceToHost, st));
    MSG_CUDA(ctx, cudaStreamSynchronize(st));
    // d_q (n3 * Rp floats >= R doubles) is free after the loop
    k_ebe_tip<<<(R + 127) / 128, 128, 0, st>>>(R, Rp, row, d_x.as<double>(), d_q.as<double>());
    count_launch(ctx);
    MSG_CUDA(ctx, cudaMemcpyAsync(out.tip, d_q.ptr, sizeof(double) * R, cudaMemcpyDeviceToHost, st));
  }
  std::vector<int> its(Rp), done(Rp);
  std::vector<double> res(Rp);
  MSG_CUDA(ctx, cudaMemcpyAsync(its.data(), s.its, sizeof(int) * Rp, cudaMemcpyDeviceToHost, st));
  MSG_CUDA(ctx, cudaMemcpyAsync(done.data(), s.done, sizeof(int) * Rp, cudaMemcpyDeviceToHost, st));
  MSG_CUDA(ctx, cudaMemcpyAsync(res.data(), s.res, sizeof(double) * Rp, cudaMemcpyDeviceToHost, st));
  MSG_CUDA(ctx, cudaStreamSynchronize(st));
  MSG_CUDA(ctx, cudaGetLastError());
  int status = MSG_OK;
  for (int r = 0; r < R; ++r) {
    if (out.iterations) out.iterations[r] = its[r];
    if (out.rel_res) out.rel_res[r] = res[r];
    if (done[r] != 1 && status == MSG_OK) status = done[r] == 2 ? MSG_ERR_BREAKDOWN : MSG_ERR_NOT_CONVERGED;
  }
  if (status != MSG_OK) set_error(ctx, status, "element-by-element batch: a realization did not converge");
  return status;
}

}  // namespace msg
