// Batched mixed-precision Monte Carlo solves on any Hexa8 meshes (distorted,
// unstructured, and of different sizes in one batch): the path of
// MonteCarloAnalyzerWithStochasticMaterial.SolveNormal
// (ISAAR.MSolve.Analyzers/MonteCarloAnalyzerWithStochasticMaterial.cs:232-296)
// for all realizations of several systems at once, where the cube-lattice
// operators do not apply.
//
// Operator. The stiffness of element e in realization r is K_e = E_{e,r} Khat_e
// with Khat_e the element's stiffness at E = 1 (the constitutive matrix is
// linear in E; Hexa8WithStochasticMaterial.cs:61-110 evaluates E once per
// element), so Khat_e is computed once per mesh and shared by every
// realization. The operator is applied node by node: the rows of node n are
//   y_n = sum over the elements e around n (corner a of e) of
//         E_{e,r} Khat_e[3a .. 3a+2][0 .. 23] u_e,
// one warp per node and up to 8 groups of 32 realizations (realization
// innermost, every vector access one 128-byte line). The 72 values of the
// corner's rows are broadcast loads shared by the groups. Each output is
// written once and the sums over the elements run in a fixed order: no
// atomics, deterministic results.
//
// Batch. A batch is a list of systems (mesh, E field, realizations, load);
// every node-level launch walks one list of work items (system, block of 64
// nodes, range of realizations) with persistent CTAs, so systems of uneven
// size share every launch. Per-realization sums go through [block][Rp]
// partial arrays of their system, added in block order by one warp per
// realization.
//
// Loop (Jacobi-preconditioned CG per realization, SolverPCG.cs:105-149 with
// the reference's diagonal preconditioner), three launches an iteration:
//   operator:  q = K p (FP32) and the partials p.q (FP64), (D r).q, q.D.q (FP32
//              within a warp);
//   scalars:   alpha = gamma / p.q and the next gamma by the expansion
//              (D r').r' = gamma - 2 alpha (D r).q + alpha^2 q.D.q, so that
//              beta is known before the update pass;
//   update:    d += alpha p, r -= alpha q, p = D r + beta p with the exact
//              partials (D r).r and r.r of the new residual (the next
//              iteration's gamma and the convergence checks).
// The iterate is x (FP64) plus an FP32 correction d. A realization asks for a
// true residual when its recursive ||r|| has dropped by `reliable_delta` since
// its last one, or below tol ||b|| / 2, or at the iteration limit; at the end
// of the 8-iteration chunk (one CUDA graph launch) every running realization
// of a system where one asked folds d into x and replaces r by the FP64
// r = b - K x (the FP64 operator); those below tol stop, the others continue
// from the true residual with their directions kept. Only those systems take
// part, so a system's arithmetic is independent of the rest of the batch: it
// gives the same bits alone and in any mix.
#include <algorithm>
#include <chrono>
#include <memory>
#include <vector>

#include "msg_internal.h"

namespace msg {
namespace {

constexpr int kEbeWarps = 8;   // warps per CTA
constexpr int kEbeCheck = 8;   // iterations per chunk (graph launch) between host reads of the flags
constexpr int kRgBlk = 64;     // nodes per work item of the operator passes: 8 warps x 8 nodes
constexpr int kRgBlkU = 256;   // nodes per work item of the update pass: 8 warps x 32 nodes
constexpr int kRgParts = 5;    // partial arrays per system over kRgBlk blocks
enum { kPq = 0, kDrq = 1, kDqd = 2, kZr = 3, kRr = 4 };

// One system of a batch (device table).
struct RgSys {
  int n_nodes, Rp, n_blk, goff;  // goff: index of realization 0 in the batch-wide scalar arrays
  int n_blk_u;                   // blocks of the update pass
  const int* inc_ptr;            // [n_nodes + 1] node -> (element, corner) incidence
  const int* inc;                // (e << 3) | a, ascending e per node
  const int* conn;               // [n_elems][8]
  const uint8_t* mask;           // [n_nodes] constrained components
  const float* K32;              // [n_elems][8][72] Khat_e per corner (FP32)
  const double* K64;             // the same in FP64
  const float* E32;              // [n_elems][Rp]
  const double* E64;
  const double* b;               // [n_nodes * 3] load (node layout)
  double* x;                     // [n_nodes * 3][Rp]
  float *d, *r, *p, *q, *dinv;   // [n_nodes * 3][Rp]
  double* part;                  // [kRgParts][n_blk][Rp]
  double* part_u;                // [2][n_blk_u][Rp]: (D r).r and r.r of the update pass (z.r, r.r: ebe_mg_solve)
  int kind;                      // ebe_mg_solve: 1 multigrid V-cycle, 0 diagonal preconditioner
  float* z;                      // ebe_mg_solve: preconditioned residual ([n_nodes * 3][Rp], or lattice layout)
  // V-cycle systems: the lattice's r buffer and the padded lattice index of
  // each node; z then is the lattice's z buffer, indexed the same way
  float* rl;
  const int* lmap;
  // V-cycle systems: z.r of the last apply, from the V-cycle's own partials
  // (lzr[(block * Rp + realization) * 2], lzr_blocks blocks)
  const double* lzr;
  int lzr_blocks;
};
struct RgItem {
  int sys, blk, rb, G;  // nodes blk * 64 .., realizations rb .. rb + 32 G - 1
};
// Batch-wide per-realization state, index = system goff + realization.
struct RgScal {
  double *gamma, *rr_ref, *bnorm, *res;
  float *alpha, *beta;
  int *done;   // 0 running, 1 converged (or padding), 2 breakdown, 3 iteration limit
  int *its;    // FP32 operator products
  int *rsys;   // system of the realization
  int *sreq;   // per system: 1 when one of its realizations asked for a true residual
  int *gact;   // per group of 32 realizations: 1 while one of them runs
  int* flags;  // [0] requests in this chunk, [1] realizations still running
};

// Whether the work item has a running realization (the same for the whole CTA).
__device__ __forceinline__ bool rg_item_active(const int* __restrict__ gact, int goff, int rb, int G) {
  bool a = false;
  for (int g = 0; g < G; ++g) a |= gact[(goff + rb) / 32 + g] != 0;
  return a;
}

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

// CTA sum (fixed warp order) of the lanes' values into dst[lane].
__device__ __forceinline__ void rg_block_partial(double v, double* sh, double* __restrict__ dst) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  sh[w * 32 + lane] = v;
  __syncthreads();
  if (w == 0) {
    double s = 0.0;
    for (int i = 0; i < kEbeWarps; ++i) s += sh[i * 32 + lane];
    dst[lane] = s;
  }
  __syncthreads();
}

// The same for N values per lane with one barrier pair: value i of every lane
// into dst(i)[lane], warps added in the same fixed order.
template <int N, class T, int M, class Dst>
__device__ __forceinline__ void rg_block_partials(const T (&v)[N], double (&sh)[M], Dst dst) {
  static_assert(M >= N * kEbeWarps * 32, "shared buffer of rg_block_partials");
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int i = 0; i < N; ++i) sh[(i * kEbeWarps + w) * 32 + lane] = (double)v[i];
  __syncthreads();
  for (int j = threadIdx.x; j < N * 32; j += blockDim.x) {
    const int i = j >> 5, l = j & 31;
    double t = 0.0;
    for (int k = 0; k < kEbeWarps; ++k) t += sh[(i * kEbeWarps + k) * 32 + l];
    dst(i)[l] = t;
  }
  __syncthreads();
}

__device__ __forceinline__ double* rg_part(const RgSys& S, int k, int blk, int col) {
  return S.part + ((size_t)k * S.n_blk + blk) * S.Rp + col;
}

// Node rows of K u in FP32 for G realization groups of 32 (realizations
// rb + 32 g + lane): the corner's 72 values as 18 float4 broadcast loads (each
// per-corner block starts on a 288-byte boundary), used by all G groups. A
// broadcast load fills 32 lanes' registers, so its cost in the load
// writeback path is shared by the G groups. Each gathered u value is scaled
// by the element's E first (E_e Khat_e u_e = Khat_e (E_e u_e)), so the sum
// over the element runs straight into y and no per-element partial sums are
// held. Every realization's arithmetic (order of the products and sums) is
// the same for every G.
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
    float Ee[G];
#pragma unroll
    for (int g = 0; g < G; ++g) Ee[g] = E[(size_t)e * Rp + rb + 32 * g + lane];
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
          const float uv = Ee[g] * ub[32 * g];
          y[g][0] = fmaf(kv[3 * s], uv, y[g][0]);
          y[g][1] = fmaf(kv[3 * s + 1], uv, y[g][1]);
          y[g][2] = fmaf(kv[3 * s + 2], uv, y[g][2]);
        }
      }
    }
  }
}

// The node rows in FP64 for G realization groups (true residuals), the
// corner's values loaded once for the G groups.
template <int G>
__device__ __forceinline__ void ebe_rows64(int n, int Rp, int rb, const int* __restrict__ inc_ptr,
                                           const int* __restrict__ inc, const int* __restrict__ conn,
                                           const double* __restrict__ Kh, const double* __restrict__ E,
                                           const double* __restrict__ u, double (&y)[G][3]) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int g = 0; g < G; ++g) y[g][0] = y[g][1] = y[g][2] = 0.0;
  const int k1 = __ldg(inc_ptr + n + 1);
  for (int k = __ldg(inc_ptr + n); k < k1; ++k) {
    const int ea = __ldg(inc + k);
    const int e = ea >> 3, a = ea & 7;
    const double2* __restrict__ K2 = reinterpret_cast<const double2*>(Kh + (size_t)e * 576 + 72 * a);
    const int4 c0 = __ldg(reinterpret_cast<const int4*>(conn) + 2 * (size_t)e);
    const int4 c1 = __ldg(reinterpret_cast<const int4*>(conn) + 2 * (size_t)e + 1);
    const int nb[8] = {c0.x, c0.y, c0.z, c0.w, c1.x, c1.y, c1.z, c1.w};
    double t[G][3];
#pragma unroll
    for (int g = 0; g < G; ++g) t[g][0] = t[g][1] = t[g][2] = 0.0;
#pragma unroll
    for (int q = 0; q < 12; ++q) {  // 2 columns (3 double2, 6 values) per step
      const double2 ka = __ldg(K2 + 3 * q), kb = __ldg(K2 + 3 * q + 1), kc = __ldg(K2 + 3 * q + 2);
      const int j0 = 2 * q, j1 = 2 * q + 1;
      const double* __restrict__ u0p = u + ((size_t)nb[j0 / 3] * 3 + j0 % 3) * Rp + rb + lane;
      const double* __restrict__ u1p = u + ((size_t)nb[j1 / 3] * 3 + j1 % 3) * Rp + rb + lane;
#pragma unroll
      for (int g = 0; g < G; ++g) {
        const double u0 = u0p[32 * g], u1 = u1p[32 * g];
        t[g][0] = fma(ka.x, u0, t[g][0]);
        t[g][1] = fma(ka.y, u0, t[g][1]);
        t[g][2] = fma(kb.x, u0, t[g][2]);
        t[g][0] = fma(kb.y, u1, t[g][0]);
        t[g][1] = fma(kc.x, u1, t[g][1]);
        t[g][2] = fma(kc.y, u1, t[g][2]);
      }
    }
#pragma unroll
    for (int g = 0; g < G; ++g) {
      const double Ee = E[(size_t)e * Rp + rb + 32 * g + lane];
      y[g][0] = fma(Ee, t[g][0], y[g][0]);
      y[g][1] = fma(Ee, t[g][1], y[g][1]);
      y[g][2] = fma(Ee, t[g][2], y[g][2]);
    }
  }
}

// ---------------------------------------------------------------- loop kernels (work items)

// q = K p (FP32, constrained components 0) and the partials p.q, (D r).q, q.D.q.
template <int G>
__device__ __forceinline__ void rg_apply_item(const RgSys& S, int blk, int rb, double* sh, bool pq_only) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int Rp = S.Rp;
  // p.q (alpha) in FP64; (D r).q and q.D.q, which only enter beta's estimate, in
  // FP32 within a warp (FP64 across the warps and blocks)
  double pq[G];
  float drq[G], dqd[G];
#pragma unroll
  for (int g = 0; g < G; ++g) {
    pq[g] = 0.0;
    drq[g] = dqd[g] = 0.f;
  }
  const int n1 = min(S.n_nodes, (blk + 1) * kRgBlk);
  for (int n = blk * kRgBlk + w; n < n1; n += kEbeWarps) {
    float y[G][3];
    ebe_rows32<G>(n, Rp, rb, S.inc_ptr, S.inc, S.conn, S.K32, S.E32, S.p, y);
    const unsigned mk = __ldg(S.mask + n);
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int g = 0; g < G; ++g) {
        const size_t o = ((size_t)n * 3 + c) * Rp + rb + 32 * g + lane;
        const float v = ((mk >> c) & 1u) ? 0.f : y[g][c];
        S.q[o] = v;
        pq[g] += (double)S.p[o] * (double)v;
        if (!pq_only) {
          const float dv = S.dinv[o];
          drq[g] = fmaf(dv * S.r[o], v, drq[g]);
          dqd[g] = fmaf(dv * v, v, dqd[g]);
        }
      }
  }
  // one value at a time: three arrays of G live across one barrier spill under
  // the 128-register cap
#pragma unroll
  for (int g = 0; g < G; ++g) {
    rg_block_partial(pq[g], sh, rg_part(S, kPq, blk, rb + 32 * g));
    if (!pq_only) {
      rg_block_partial((double)drq[g], sh, rg_part(S, kDrq, blk, rb + 32 * g));
      rg_block_partial((double)dqd[g], sh, rg_part(S, kDqd, blk, rb + 32 * g));
    }
  }
}

// Every G in one kernel at 128 registers a thread (2 CTAs an SM): each
// variant gets registers for many gathers in flight. Compiled alone, G = 4
// takes 80 registers (3 CTAs an SM) and runs 24 % slower at 32^3 x 512.
// pq_only (the standard PCG of ebe_mg_solve): p.q alone, without the partials
// of beta's expansion and their reads of r and D^-1.
__global__ void __launch_bounds__(32 * kEbeWarps, 2) k_rg_apply(const RgSys* __restrict__ Sys,
                                                            const RgItem* __restrict__ items, int n_items,
                                                            const int* __restrict__ gact, int pq_only) {
  __shared__ double sh[kEbeWarps * 32];
  for (int it = blockIdx.x; it < n_items; it += gridDim.x) {
    const RgItem I = items[it];
    const RgSys S = Sys[I.sys];
    if (!rg_item_active(gact, S.goff, I.rb, I.G)) continue;
    switch (I.G) {
      case 8: rg_apply_item<8>(S, I.blk, I.rb, sh, pq_only != 0); break;
      case 4: rg_apply_item<4>(S, I.blk, I.rb, sh, pq_only != 0); break;
      case 2: rg_apply_item<2>(S, I.blk, I.rb, sh, pq_only != 0); break;
      default: rg_apply_item<1>(S, I.blk, I.rb, sh, pq_only != 0);
    }
  }
}

// d += alpha p, r -= alpha q, p = D r + beta p; partials (D r).r and r.r. A
// memory-bound pass with nothing to share between realization groups: work
// items of 256 nodes and one group, one CTA each (few registers, long streams
// per warp, two nodes in flight); items of groups without a running
// realization skipped.
__global__ void __launch_bounds__(32 * kEbeWarps) k_rg_update(const RgSys* __restrict__ Sys,
                                                             const RgItem* __restrict__ items, int n_items,
                                                             RgScal s) {
  __shared__ double sh[2 * kEbeWarps * 32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int it = blockIdx.x; it < n_items; it += gridDim.x) {
    const RgItem I = items[it];
    const RgSys S = Sys[I.sys];
    if (!s.gact[(S.goff + I.rb) / 32]) continue;  // the same for the whole CTA
    const int Rp = S.Rp, col = I.rb;
    const int n1 = min(S.n_nodes, (I.blk + 1) * kRgBlkU);
    const float al = s.alpha[S.goff + col + lane], be = s.beta[S.goff + col + lane];
    double zr = 0.0, rr = 0.0;
#pragma unroll 2
    for (int n = I.blk * kRgBlkU + w; n < n1; n += kEbeWarps)
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const size_t o = ((size_t)n * 3 + c) * Rp + col + lane;
        const float pv = S.p[o];
        const float rv = fmaf(-al, S.q[o], S.r[o]);
        S.d[o] = fmaf(al, pv, S.d[o]);
        const float zv = S.dinv[o] * rv;
        S.p[o] = fmaf(be, pv, zv);
        S.r[o] = rv;
        zr += (double)zv * (double)rv;
        rr += (double)rv * (double)rv;
      }
    const double v[2] = {zr, rr};
    rg_block_partials(v, sh, [&](int i) { return S.part_u + ((size_t)i * S.n_blk_u + I.blk) * Rp + col; });
  }
}

// x += d, d = 0 for the systems with a true residual pending (all = 1: every
// system; a realization's d is 0 after its last true residual).
__global__ void k_rg_fold(const RgSys* __restrict__ Sys, const RgItem* __restrict__ items, int n_items, RgScal s,
                          int all) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int it = blockIdx.x; it < n_items; it += gridDim.x) {
    const RgItem I = items[it];
    if (!all && !s.sreq[I.sys]) continue;
    const RgSys S = Sys[I.sys];
    const int n1 = min(S.n_nodes, (I.blk + 1) * kRgBlk);
    for (int g = 0; g < I.G; ++g) {
      const int col = I.rb + 32 * g + lane;
      for (int n = I.blk * kRgBlk + w; n < n1; n += kEbeWarps)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const size_t o = ((size_t)n * 3 + c) * S.Rp + col;
          S.x[o] += (double)S.d[o];
          S.d[o] = 0.f;
        }
    }
  }
}

// FP64 true residual r = b - K x (constrained components 0) of every
// realization of the systems with a true residual pending, into r (FP32);
// partials r.r and (D r).r. The item's groups two at a time.
template <int G>
__device__ __forceinline__ void rg_resid_groups(const RgSys& S, int blk, int rb, double* sh) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  double s_rr[G], s_zr[G];
#pragma unroll
  for (int g = 0; g < G; ++g) s_rr[g] = s_zr[g] = 0.0;
  const int n1 = min(S.n_nodes, (blk + 1) * kRgBlk);
  for (int n = blk * kRgBlk + w; n < n1; n += kEbeWarps) {
    double y[G][3];
    ebe_rows64<G>(n, S.Rp, rb, S.inc_ptr, S.inc, S.conn, S.K64, S.E64, S.x, y);
    const unsigned mk = __ldg(S.mask + n);
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int g = 0; g < G; ++g) {
        const size_t o = ((size_t)n * 3 + c) * S.Rp + rb + 32 * g + lane;
        const double v = ((mk >> c) & 1u) ? 0.0 : S.b[(size_t)n * 3 + c] - y[g][c];
        const float v32 = (float)v;
        S.r[o] = v32;
        s_rr[g] += v * v;
        s_zr[g] += (double)(S.dinv[o] * v32) * (double)v32;
      }
  }
#pragma unroll
  for (int g = 0; g < G; ++g) {
    rg_block_partial(s_rr[g], sh, rg_part(S, kRr, blk, rb + 32 * g));
    rg_block_partial(s_zr[g], sh, rg_part(S, kZr, blk, rb + 32 * g));
  }
}

__global__ void __launch_bounds__(32 * kEbeWarps) k_rg_resid64(const RgSys* __restrict__ Sys,
                                                              const RgItem* __restrict__ items, int n_items,
                                                              RgScal s) {
  __shared__ double sh[kEbeWarps * 32];
  for (int it = blockIdx.x; it < n_items; it += gridDim.x) {
    const RgItem I = items[it];
    if (!s.sreq[I.sys]) continue;  // the same for the whole CTA
    const RgSys S = Sys[I.sys];
    if (I.G == 4) {  // four groups to an element-row load when all four run
      const int grp = (S.goff + I.rb) / 32;
      if (s.gact[grp] && s.gact[grp + 1] && s.gact[grp + 2] && s.gact[grp + 3]) {
        rg_resid_groups<4>(S, I.blk, I.rb, sh);
        continue;
      }
    }
    for (int g = 0; g < I.G; g += 2) {
      const int grp = (S.goff + I.rb) / 32 + g;
      const bool a0 = s.gact[grp] != 0, a1 = g + 1 < I.G && s.gact[grp + 1] != 0;
      if (a0 && a1)
        rg_resid_groups<2>(S, I.blk, I.rb + 32 * g, sh);
      else if (a0)
        rg_resid_groups<1>(S, I.blk, I.rb + 32 * g, sh);
      else if (a1)
        rg_resid_groups<1>(S, I.blk, I.rb + 32 * (g + 1), sh);
    }
  }
}

// ---------------------------------------------------------------- per-realization scalars (one warp each)

// Sum over the block partials of realization r by one warp: lane l adds blocks
// l, l + 32, ... in order, then a butterfly over the lanes (every lane gets the
// same bits: each step adds the same two values on both lanes of a pair).
__device__ __forceinline__ double rg_sum(const double* __restrict__ part, int n_blk, int Rp, int r) {
  const int lane = threadIdx.x & 31;
  double v = 0.0;
  for (int i = lane; i < n_blk; i += 32) v += part[(size_t)i * Rp + r];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// z.r of system-local realization r after z = M^-1 r: the V-cycle's partials
// (two values a block and realization, z.r the second) or the diagonal pass's
__device__ __forceinline__ double rg_sum_zr(const RgSys& S, int r) {
  if (!S.lzr) return rg_sum(S.part_u, S.n_blk_u, S.Rp, r);
  const int lane = threadIdx.x & 31;
  double v = 0.0;
  for (int i = lane; i < S.lzr_blocks; i += 32) v += S.lzr[((size_t)i * S.Rp + r) * 2];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ int rg_warp_index() { return (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5); }

// A realization asks for a true residual of its system.
__device__ __forceinline__ void rg_check(const RgScal& s, int g, double rr, double tol2, double delta2, int max_it) {
  const double b2 = s.bnorm[g] * s.bnorm[g];
  if (rr < tol2 * b2 || rr < delta2 * s.rr_ref[g] || s.its[g] >= max_it || !isfinite(rr)) {
    const int sys = s.rsys[g];
    if (!s.sreq[sys]) atomicAdd(s.flags, 1);
    s.sreq[sys] = 1;
  }
}

// alpha = gamma / p.q and beta = gamma' / gamma with gamma' by the expansion;
// consume = 1: gamma and the check from the previous update's exact partials.
__global__ void k_rg_scalar(const RgSys* __restrict__ Sys, int Rtot, RgScal s, int consume, double tol2,
                            double delta2, int max_it) {
  const int g = rg_warp_index();
  if (g >= Rtot) return;
  const int lane = threadIdx.x & 31;
  if (s.done[g]) {
    if (lane == 0) s.alpha[g] = s.beta[g] = 0.f;
    return;
  }
  const RgSys& S = Sys[s.rsys[g]];
  const int Rp = S.Rp, nb = S.n_blk, r = g - S.goff;
  const size_t P = (size_t)nb * Rp;
  double gam = s.gamma[g];
  if (consume) {
    const size_t Pu = (size_t)S.n_blk_u * Rp;
    const double zr = rg_sum(S.part_u, S.n_blk_u, Rp, r), rr = rg_sum(S.part_u + Pu, S.n_blk_u, Rp, r);
    gam = zr;
    if (lane == 0) rg_check(s, g, rr, tol2, delta2, max_it);
  }
  const double pq = rg_sum(S.part + kPq * P, nb, Rp, r);
  const double drq = rg_sum(S.part + kDrq * P, nb, Rp, r);
  const double dqd = rg_sum(S.part + kDqd * P, nb, Rp, r);
  if (lane != 0) return;
  s.its[g] += 1;
  s.gamma[g] = gam;
  if (!(gam > 0.0)) {  // r = 0: nothing to do until the true residual
    s.alpha[g] = s.beta[g] = 0.f;
    return;
  }
  if (!(pq > 0.0) || !isfinite(pq)) {
    s.done[g] = 2;
    s.alpha[g] = s.beta[g] = 0.f;
    return;
  }
  const float af = (float)(gam / pq);
  const double a = (double)af;
  const double est = gam - 2.0 * a * drq + a * a * dqd;
  s.alpha[g] = af;
  s.beta[g] = est > 0.0 ? (float)(est / gam) : 0.f;
}

// End of a chunk: gamma and the check from the last update's partials;
// flags[1] counts the realizations still running.
__global__ void k_rg_chunk_end(const RgSys* __restrict__ Sys, int Rtot, RgScal s, double tol2, double delta2,
                               int max_it) {
  const int g = rg_warp_index();
  if (g >= Rtot || s.done[g]) return;
  const RgSys& S = Sys[s.rsys[g]];
  const int Rp = S.Rp, r = g - S.goff;
  const size_t Pu = (size_t)S.n_blk_u * Rp;
  const double zr = rg_sum(S.part_u, S.n_blk_u, Rp, r), rr = rg_sum(S.part_u + Pu, S.n_blk_u, Rp, r);
  if ((threadIdx.x & 31) != 0) return;
  s.gamma[g] = zr;
  rg_check(s, g, rr, tol2, delta2, max_it);
  atomicAdd(s.flags + 1, 1);
}

// After the FP64 true residual: a realization of a system with a true
// residual stops below tol (or at the iteration limit) or continues from the
// true residual; flags[1] counts the realizations still running.
__global__ void k_rg_true(const RgSys* __restrict__ Sys, int Rtot, RgScal s, double tol, int max_it) {
  const int g = rg_warp_index();
  if (g >= Rtot || s.done[g]) return;
  const int lane = threadIdx.x & 31;
  if (!s.sreq[s.rsys[g]]) {
    if (lane == 0) atomicAdd(s.flags + 1, 1);
    return;
  }
  const RgSys& S = Sys[s.rsys[g]];
  const int Rp = S.Rp, nb = S.n_blk, r = g - S.goff;
  const size_t P = (size_t)nb * Rp;
  const double rr = rg_sum(S.part + kRr * P, nb, Rp, r), zr = rg_sum(S.part + kZr * P, nb, Rp, r);
  if (lane != 0) return;
  const double err = s.bnorm[g] > 0.0 ? sqrt(rr) / s.bnorm[g] : 0.0;
  s.res[g] = err;
  s.rr_ref[g] = rr;
  s.gamma[g] = zr;
  if (err < tol) {
    s.done[g] = 1;
  } else if (s.its[g] >= max_it || !isfinite(err)) {
    s.done[g] = 3;
  } else {
    atomicAdd(s.flags + 1, 1);
  }
}

// flags[1] = realizations still running (the multigrid-preconditioned loop's chunk end).
__global__ void k_rg_chunk_end_count(int Rtot, RgScal s) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g < Rtot && !s.done[g]) atomicAdd(s.flags + 1, 1);
}

// gact[group] = 1 while one of the group's 32 realizations runs (one warp per group).
__global__ void k_rg_active(int n_groups, RgScal s) {
  const int grp = rg_warp_index();
  if (grp >= n_groups) return;
  const unsigned run = __ballot_sync(0xffffffffu, s.done[grp * 32 + (threadIdx.x & 31)] == 0);
  if ((threadIdx.x & 31) == 0) s.gact[grp] = run != 0u;
}

// ---------------------------------------------------------------- per-system setup and results

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

// x = 0, d = 0, r = b, p = D b; partials (D b).b and b.b. Grid (n_blk, Rp / 32).
__global__ void __launch_bounds__(32 * kEbeWarps) k_rg_init(RgSys S) {
  __shared__ double sh[kEbeWarps * 32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int blk = blockIdx.x, col = blockIdx.y * 32 + lane;
  const int n1 = min(S.n_nodes, (blk + 1) * kRgBlk);
  double s_zr = 0.0, s_rr = 0.0;
  for (int n = blk * kRgBlk + w; n < n1; n += kEbeWarps)
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const size_t o = ((size_t)n * 3 + c) * S.Rp + col;
      const double bd = S.b[(size_t)n * 3 + c];
      const float bv = (float)bd;
      const float zv = S.dinv[o] * bv;
      S.x[o] = 0.0;
      S.d[o] = 0.f;
      S.r[o] = bv;
      S.p[o] = zv;
      s_zr += (double)zv * (double)bv;
      s_rr += bd * bd;
    }
  rg_block_partial(s_zr, sh, rg_part(S, kZr, blk, blockIdx.y * 32));
  rg_block_partial(s_rr, sh, rg_part(S, kRr, blk, blockIdx.y * 32));
}

// Starting scalars of one system's realizations (one warp each); a zero load
// (and padding) is done at once with x = 0.
__global__ void k_rg_start(RgSys S, int R, RgScal s) {
  const int r = rg_warp_index();
  if (r >= S.Rp) return;
  const size_t P = (size_t)S.n_blk * S.Rp;
  const double bb = rg_sum(S.part + kRr * P, S.n_blk, S.Rp, r), zr = rg_sum(S.part + kZr * P, S.n_blk, S.Rp, r);
  if ((threadIdx.x & 31) != 0) return;
  const int g = S.goff + r;
  s.bnorm[g] = sqrt(bb);
  s.rr_ref[g] = bb;
  s.gamma[g] = zr;
  s.alpha[g] = s.beta[g] = 0.f;
  s.its[g] = 0;
  s.res[g] = bb > 0.0 ? 1.0 : 0.0;
  s.done[g] = (r >= R || !(bb > 0.0)) ? 1 : 0;
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

// ---------------------------------------------------------------- preconditioned loop (V-cycle or diagonal per system)
// Standard PCG with z = M^-1 r: M^-1 the V-cycle of the system's cube lattice
// (gmg_precond_apply) or the diagonal (k_vc_jacobi_z):
// operator (k_rg_apply: q = K p, partial p.q), alpha, update (r, d and r.r),
// preconditioner, z.r, beta, direction. Work items of the update pass; the
// partials of the update pass are part_u [0] z.r and [1] r.r.

// r -= alpha q, d += alpha p, partial r.r (into part_u[1])
__global__ void __launch_bounds__(32 * kEbeWarps) k_vc_update(const RgSys* __restrict__ Sys,
                                                             const RgItem* __restrict__ items, int n_items,
                                                             RgScal s) {
  __shared__ double sh[kEbeWarps * 32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int it = blockIdx.x; it < n_items; it += gridDim.x) {
    const RgItem I = items[it];
    const RgSys S = Sys[I.sys];
    if (!s.gact[(S.goff + I.rb) / 32]) continue;  // the same for the whole CTA
    const int Rp = S.Rp, col = I.rb;
    const int n1 = min(S.n_nodes, (I.blk + 1) * kRgBlkU);
    const float al = s.alpha[S.goff + col + lane];
    double rr = 0.0;
#pragma unroll 2
    for (int n = I.blk * kRgBlkU + w; n < n1; n += kEbeWarps)
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const size_t o = ((size_t)n * 3 + c) * Rp + col + lane;
        const float rv = fmaf(-al, S.q[o], S.r[o]);
        S.d[o] = fmaf(al, S.p[o], S.d[o]);
        S.r[o] = rv;
        if (S.lmap) S.rl[((size_t)__ldg(S.lmap + n) * 3 + c) * Rp + col + lane] = rv;  // the V-cycle's input
        rr += (double)rv * (double)rv;
      }
    rg_block_partial(rr, sh, S.part_u + ((size_t)1 * S.n_blk_u + I.blk) * Rp + col);
  }
}

// p = z + beta p
__global__ void __launch_bounds__(32 * kEbeWarps) k_vc_dir(const RgSys* __restrict__ Sys, const RgItem* __restrict__ items,
                                                          int n_items, RgScal s) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int it = blockIdx.x; it < n_items; it += gridDim.x) {
    const RgItem I = items[it];
    const RgSys S = Sys[I.sys];
    if (!s.gact[(S.goff + I.rb) / 32]) continue;
    const int Rp = S.Rp, col = I.rb;
    const int n1 = min(S.n_nodes, (I.blk + 1) * kRgBlkU);
    const float be = s.beta[S.goff + col + lane];
#pragma unroll 2
    for (int n = I.blk * kRgBlkU + w; n < n1; n += kEbeWarps)
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const size_t o = ((size_t)n * 3 + c) * Rp + col + lane;
        const size_t oz = S.lmap ? ((size_t)__ldg(S.lmap + n) * 3 + c) * Rp + col + lane : o;
        S.p[o] = fmaf(be, S.p[o], S.z[oz]);
      }
  }
}

// z = D^-1 r and the partial z.r (into part_u[0]) for the systems with the
// diagonal preconditioner; the V-cycle writes its own z.r partials
__global__ void __launch_bounds__(32 * kEbeWarps) k_vc_jacobi_z(const RgSys* __restrict__ Sys,
                                                               const RgItem* __restrict__ items, int n_items,
                                                               RgScal s) {
  __shared__ double sh[kEbeWarps * 32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int it = blockIdx.x; it < n_items; it += gridDim.x) {
    const RgItem I = items[it];
    const RgSys S = Sys[I.sys];
    if (S.kind != 0 || !s.gact[(S.goff + I.rb) / 32]) continue;
    const int Rp = S.Rp, col = I.rb;
    const int n1 = min(S.n_nodes, (I.blk + 1) * kRgBlkU);
    double zr = 0.0;
#pragma unroll 2
    for (int n = I.blk * kRgBlkU + w; n < n1; n += kEbeWarps)
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const size_t o = ((size_t)n * 3 + c) * Rp + col + lane;
        const float rv = S.r[o], zv = S.dinv[o] * rv;
        S.z[o] = zv;
        zr += (double)zv * (double)rv;
      }
    rg_block_partial(zr, sh, S.part_u + (size_t)I.blk * Rp + col);
  }
}

// alpha = gamma / p.q (one warp per realization)
__global__ void k_vc_alpha(const RgSys* __restrict__ Sys, int Rtot, RgScal s) {
  const int g = rg_warp_index();
  if (g >= Rtot) return;
  const int lane = threadIdx.x & 31;
  if (s.done[g]) {
    if (lane == 0) s.alpha[g] = 0.f;
    return;
  }
  const RgSys& S = Sys[s.rsys[g]];
  const int r = g - S.goff;
  const double pq = rg_sum(S.part + (size_t)kPq * S.n_blk * S.Rp, S.n_blk, S.Rp, r);
  if (lane != 0) return;
  s.its[g] += 1;
  if (!(pq > 0.0) || !isfinite(pq)) {
    s.done[g] = 2;
    s.alpha[g] = 0.f;
    return;
  }
  s.alpha[g] = (float)(s.gamma[g] / pq);
}

// beta = gamma_new / gamma with gamma_new = z.r, and the true-residual check on r.r
__global__ void k_vc_beta(const RgSys* __restrict__ Sys, int Rtot, RgScal s, double tol2, double delta2,
                          int max_it) {
  const int g = rg_warp_index();
  if (g >= Rtot) return;
  const int lane = threadIdx.x & 31;
  if (s.done[g]) {
    if (lane == 0) s.beta[g] = 0.f;
    return;
  }
  const RgSys& S = Sys[s.rsys[g]];
  const int r = g - S.goff;
  const size_t Pu = (size_t)S.n_blk_u * S.Rp;
  const double zr = rg_sum_zr(S, r), rr = rg_sum(S.part_u + Pu, S.n_blk_u, S.Rp, r);
  if (lane != 0) return;
  s.beta[g] = s.gamma[g] > 0.0 ? (float)(zr / s.gamma[g]) : 0.f;
  s.gamma[g] = zr;
  rg_check(s, g, rr, tol2, delta2, max_it);
}

// Starting scalars: ||b|| from the init partials, gamma = z.b, beta = 0 (p = z)
__global__ void k_vc_start(RgSys S, int R, RgScal s) {
  const int r = rg_warp_index();
  if (r >= S.Rp) return;
  const double bb = rg_sum(S.part + (size_t)kRr * S.n_blk * S.Rp, S.n_blk, S.Rp, r);
  const double zr = rg_sum_zr(S, r);
  if ((threadIdx.x & 31) != 0) return;
  const int g = S.goff + r;
  s.bnorm[g] = sqrt(bb);
  s.rr_ref[g] = bb;
  s.gamma[g] = zr;
  s.alpha[g] = s.beta[g] = 0.f;
  s.its[g] = 0;
  s.res[g] = bb > 0.0 ? 1.0 : 0.0;
  s.done[g] = (r >= R || !(bb > 0.0)) ? 1 : 0;
}

// After the FP64 true residual (r.r in part kRr) and z = M^-1 r (z.r in part_u[0])
// of the systems that asked; flags[1] counts the realizations still running
__global__ void k_vc_true(const RgSys* __restrict__ Sys, int Rtot, RgScal s, double tol, int max_it) {
  const int g = rg_warp_index();
  if (g >= Rtot || s.done[g]) return;
  const int lane = threadIdx.x & 31;
  if (!s.sreq[s.rsys[g]]) {  // its system took no true residual
    if (lane == 0) atomicAdd(s.flags + 1, 1);
    return;
  }
  const RgSys& S = Sys[s.rsys[g]];
  const int r = g - S.goff;
  const double rr = rg_sum(S.part + (size_t)kRr * S.n_blk * S.Rp, S.n_blk, S.Rp, r);
  const double zr = rg_sum_zr(S, r);
  if (lane != 0) return;
  const double err = s.bnorm[g] > 0.0 ? sqrt(rr) / s.bnorm[g] : 0.0;
  s.res[g] = err;
  s.rr_ref[g] = rr;
  s.gamma[g] = zr;
  if (err < tol) {
    s.done[g] = 1;
  } else if (s.its[g] >= max_it || !isfinite(err)) {
    s.done[g] = 3;
  } else {
    atomicAdd(s.flags + 1, 1);
  }
}

// Device buffers of one system (carved from the batch's arena).
struct RgBuf {
  int R = 0, Rp = 0, G = 1, n_blk = 0, n_blk_u = 0;
  std::vector<int> h_ptr, h_inc;  // incidence (host)
  int *ptr = nullptr, *inc = nullptr;
  double *K64 = nullptr, *E64 = nullptr, *bn = nullptr, *x = nullptr, *part = nullptr, *part_u = nullptr;
  float *K32 = nullptr, *E32 = nullptr, *d = nullptr, *r = nullptr, *p = nullptr, *q = nullptr, *dinv = nullptr;
};

// Sequential carving of one device allocation at 256-byte boundaries; a first
// pass with base == nullptr only adds up the bytes.
struct Carver {
  unsigned char* base = nullptr;
  size_t off = 0;
  template <class T> T* take(size_t n) {
    const size_t at = off;
    off += (sizeof(T) * std::max<size_t>(n, 1) + 255) / 256 * 256;
    return base ? reinterpret_cast<T*>(base + at) : nullptr;
  }
};

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

// Per-system sizes and incidence (host).
static int rg_plan(Context* ctx, const RgInput& in, RgBuf& B, int rp_multiple = 32) {
  Mesh* m = in.m;
  const int nn = m->n_nodes, ne = m->n_elems;
  if ((int64_t)ne * 8 >= ((int64_t)1 << 31) || nn <= 0 || ne <= 0 || in.R <= 0 || !in.kl || !in.d_xi || !in.d_b)
    return set_error(ctx, MSG_ERR_INVALID_ARGUMENT, "element-by-element batch: invalid system");
  if (in.tip_dof >= m->n_dofs) return set_error(ctx, MSG_ERR_INVALID_ARGUMENT, "tip_dof out of range");
  B.R = in.R;
  B.Rp = (in.R + rp_multiple - 1) / rp_multiple * rp_multiple;
  const int ng = B.Rp / 32;
  // groups per operator work item (the batch takes the smallest over its
  // systems): 4 by default (8 amortises the element rows further but needs 128
  // registers a thread: slower at 32^3 x 512)
  B.G = ng % 4 == 0 ? 4 : ng % 2 == 0 ? 2 : 1;
  if (ctx->element_groups > 0 && ng % ctx->element_groups == 0) B.G = ctx->element_groups;
  B.n_blk = (nn + kRgBlk - 1) / kRgBlk;
  B.n_blk_u = (nn + kRgBlkU - 1) / kRgBlkU;
  ebe_incidence(m, B.h_ptr, B.h_inc);
  return MSG_OK;
}

// The system's buffers in the arena.
static void rg_carve(const RgInput& in, RgBuf& B, Carver& c) {
  const int nn = in.m->n_nodes, ne = in.m->n_elems;
  const size_t n3 = 3 * (size_t)nn, nv = n3 * B.Rp;
  B.ptr = c.take<int>(B.h_ptr.size());
  B.inc = c.take<int>(B.h_inc.size());
  B.K64 = c.take<double>(576 * (size_t)ne);
  B.K32 = c.take<float>(576 * (size_t)ne);
  B.E64 = c.take<double>((size_t)ne * B.Rp);
  B.E32 = c.take<float>((size_t)ne * B.Rp);
  B.bn = c.take<double>(n3);
  B.x = c.take<double>(nv);
  B.d = c.take<float>(nv);
  B.r = c.take<float>(nv);
  B.p = c.take<float>(nv);
  B.q = c.take<float>(nv);
  B.dinv = c.take<float>(nv);
  B.part = c.take<double>(kRgParts * (size_t)B.n_blk * B.Rp);
  B.part_u = c.take<double>(2 * (size_t)B.n_blk_u * B.Rp);
}

// Per-system device setup: element matrices at E = 1 (through the packed
// scratch K300, at least 300 n_elems doubles), E field, load, Jacobi diagonal.
static int rg_setup(Context* ctx, const RgInput& in, RgBuf& B, double* K300, int* d_status) {
  Mesh* m = in.m;
  const int nn = m->n_nodes, ne = m->n_elems;
  const size_t n3 = 3 * (size_t)nn;
  cudaStream_t st = ctx->stream;
  MSG_CUDA(ctx, cudaMemcpyAsync(B.ptr, B.h_ptr.data(), sizeof(int) * B.h_ptr.size(), cudaMemcpyHostToDevice, st));
  MSG_CUDA(ctx, cudaMemcpyAsync(B.inc, B.h_inc.data(), sizeof(int) * B.h_inc.size(), cudaMemcpyHostToDevice, st));
  MSG_CUDA(ctx, cudaMemsetAsync(d_status, 0, sizeof(int), st));
  MSG_TRY(launch_h8_ke(ctx, ne, m->d_exyz.as<double>(), nullptr, 1.0, in.nu, K300, d_status));
  k_ebe_unpack<<<ne, 128, 0, st>>>(ne, K300, B.K64, B.K32);
  count_launch(ctx);
  // through the mapped flag words (word 8): no wait behind copies in flight
  int* hneg = ctx->h_flags + 8;
  MSG_TRY(publish_flags(ctx, d_status, 1, hneg, ctx->d_hflags ? ctx->d_hflags + 8 : nullptr, st));
  MSG_CUDA(ctx, cudaStreamSynchronize(st));
  if (*hneg) return set_error(ctx, MSG_ERR_NEG_DET, "element with a non-positive Jacobian determinant");
  // E of every element and realization [e][Rp] (the KL workspace is reused by the next system)
  KLDevice kd;
  MSG_TRY(kl_prepare(ctx, m, in.kl, &kd));
  MSG_TRY(launch_kl_field(ctx, m, &kd, in.R, B.Rp, in.d_xi, B.E64, B.E32, nullptr));
  MSG_CUDA(ctx, cudaMemsetAsync(B.bn, 0, sizeof(double) * n3, st));
  MSG_TRY(launch_dof_to_node(ctx, m, in.d_b, B.bn, 1, 0, 0));
  k_ebe_dinv<<<nn, 128, 0, st>>>(nn, B.Rp, B.ptr, B.inc, B.K64, B.E64, m->d_mask.as<uint8_t>(), B.dinv);
  count_launch(ctx);
  MSG_CUDA(ctx, cudaGetLastError());
  return MSG_OK;
}

// Results of a batch: displacements gathered into each system's X, tip values,
// iterations and residuals; the worst status.
static int rg_results(Context* ctx, const std::vector<RgInput>& in, const std::vector<RgBuf>& bufs,
                      const std::vector<RgSys>& sys, const RgScal& s, int Rtot) {
  cudaStream_t st = ctx->stream;
  const int S = (int)in.size();
  std::vector<int> its(Rtot), done(Rtot);
  std::vector<double> res(Rtot);
  MSG_CUDA(ctx, cudaMemcpyAsync(its.data(), s.its, sizeof(int) * Rtot, cudaMemcpyDeviceToHost, st));
  MSG_CUDA(ctx, cudaMemcpyAsync(done.data(), s.done, sizeof(int) * Rtot, cudaMemcpyDeviceToHost, st));
  MSG_CUDA(ctx, cudaMemcpyAsync(res.data(), s.res, sizeof(double) * Rtot, cudaMemcpyDeviceToHost, st));
  int status = MSG_OK;
  for (int i = 0; i < S; ++i) {
    const RgInput& I = in[i];
    const RgBuf& B = bufs[i];
    Mesh* m = I.m;
    if (I.d_X && m->n_dofs > 0) {
      const dim3 g((m->n_dofs + 31) / 32, B.Rp / 32);
      k_ebe_gather<<<g, dim3(32, 8), 0, st>>>(m->n_dofs, I.R, B.Rp, m->d_free_rows.as<int>(), B.x, I.d_X);
      count_launch(ctx);
    }
    if (I.h_tip && I.tip_dof >= 0) {
      int row = 0;
      MSG_CUDA(ctx, cudaMemcpyAsync(&row, m->d_free_rows.as<int>() + I.tip_dof, sizeof(int), cudaMemcpyDeviceToHost, st));
      MSG_CUDA(ctx, cudaStreamSynchronize(st));
      // q (n3 * Rp floats >= R doubles) is free after the loop
      double* tipbuf = reinterpret_cast<double*>(B.q);
      k_ebe_tip<<<(I.R + 127) / 128, 128, 0, st>>>(I.R, B.Rp, row, B.x, tipbuf);
      count_launch(ctx);
      MSG_CUDA(ctx, cudaMemcpyAsync(I.h_tip, tipbuf, sizeof(double) * I.R, cudaMemcpyDeviceToHost, st));
    }
  }
  MSG_CUDA(ctx, cudaStreamSynchronize(st));
  MSG_CUDA(ctx, cudaGetLastError());
  for (int i = 0; i < S; ++i) {
    const int g0 = sys[i].goff;
    for (int r = 0; r < in[i].R; ++r) {
      if (in[i].h_its) in[i].h_its[r] = its[g0 + r];
      if (in[i].h_res) in[i].h_res[r] = res[g0 + r];
      if (done[g0 + r] != 1 && status == MSG_OK)
        status = done[g0 + r] == 2 ? MSG_ERR_BREAKDOWN : MSG_ERR_NOT_CONVERGED;
    }
  }
  if (status != MSG_OK) set_error(ctx, status, "element-by-element batch: a realization did not converge");
  return status;
}

// The device state of an element-by-element batch: each system's buffers
// carved from one arena (workspace slot 34, kept by the context between calls;
// slot 35: the packed element matrices of one system at a time), the system
// table, the work items and the per-realization scalars.
struct RgBatch {
  int S = 0, Rtot = 0, n_items = 0, n_items_u = 0;
  std::vector<RgBuf> bufs;
  std::vector<RgSys> sys;
  std::vector<RgItem> items, items_u;
  std::vector<int> rsys;
  std::vector<float*> z;  // z [n_nodes * 3][Rp] of the systems that asked for one
  RgSys* d_sys = nullptr;
  RgItem *d_items = nullptr, *d_items_u = nullptr;
  unsigned char* scal_base = nullptr;
  int* d_status = nullptr;
  double* k300 = nullptr;
  RgScal s;
};

// Plan and carve a batch: per-system sizes (Rp a multiple of rp_multiple[i]),
// one realization-group count G for all systems (the smallest of theirs; each
// divides the next), the work items (per system and node block, the
// realization ranges one after another: operator passes 64 nodes and G groups,
// the update 256 nodes and one group, so that CTAs running at the same time
// cover whole rows [node * 3 + c][0 .. Rp) of the vectors) and the arena, with
// a z vector for each system with want_z[i].
static int rg_batch_plan(Context* ctx, const std::vector<RgInput>& in, const std::vector<int>& rp_multiple,
                         const std::vector<int>& want_z, RgBatch& b) {
  const int S = (int)in.size();
  b.S = S;
  b.bufs.assign(S, RgBuf());
  b.sys.assign(S, RgSys());
  b.z.assign(S, nullptr);
  b.Rtot = 0;
  int max_ne = 0;
  for (int i = 0; i < S; ++i) {
    if (!in[i].m || in[i].m->ctx != ctx)
      return set_error(ctx, MSG_ERR_INVALID_ARGUMENT, "element-by-element batch: system %d has no mesh of this context", i);
    MSG_TRY(rg_plan(ctx, in[i], b.bufs[i], rp_multiple[i]));
    b.sys[i].goff = b.Rtot;
    b.Rtot += b.bufs[i].Rp;
    max_ne = std::max(max_ne, in[i].m->n_elems);
  }
  int G = 8;
  for (int i = 0; i < S; ++i) G = std::min(G, b.bufs[i].G);
  for (int i = 0; i < S; ++i) b.bufs[i].G = G;
  b.items.clear();
  b.items_u.clear();
  b.rsys.assign(b.Rtot, 0);
  for (int i = 0; i < S; ++i) {
    const RgBuf& B = b.bufs[i];
    for (int blk = 0; blk < B.n_blk; ++blk)
      for (int rb = 0; rb < B.Rp; rb += 32 * B.G) b.items.push_back(RgItem{i, blk, rb, B.G});
    for (int blk = 0; blk < B.n_blk_u; ++blk)
      for (int rb = 0; rb < B.Rp; rb += 32) b.items_u.push_back(RgItem{i, blk, rb, 1});
    for (int r = 0; r < B.Rp; ++r) b.rsys[b.sys[i].goff + r] = i;
  }
  b.n_items = (int)b.items.size();
  b.n_items_u = (int)b.items_u.size();
  const size_t scal_bytes = (sizeof(double) * 4 + sizeof(float) * 2 + sizeof(int) * 3) * (size_t)b.Rtot +
                            sizeof(int) * (S + b.Rtot / 32 + 2);
  auto carve_all = [&](Carver& c) {
    for (int i = 0; i < S; ++i) {
      rg_carve(in[i], b.bufs[i], c);
      if (want_z[i]) b.z[i] = c.take<float>(3 * (size_t)in[i].m->n_nodes * b.bufs[i].Rp);
    }
    b.d_sys = c.take<RgSys>(S);
    b.d_items = c.take<RgItem>(b.items.size());
    b.d_items_u = c.take<RgItem>(b.items_u.size());
    b.scal_base = c.take<unsigned char>(scal_bytes);
    b.d_status = c.take<int>(1);
  };
  Carver count;
  carve_all(count);
  void *arena = nullptr, *k300 = nullptr;
  MSG_TRY(workspace(ctx, 34, count.off, &arena));
  MSG_TRY(workspace(ctx, 35, sizeof(double) * 300 * (size_t)max_ne, &k300));
  b.k300 = static_cast<double*>(k300);
  Carver c;
  c.base = static_cast<unsigned char*>(arena);
  carve_all(c);
  return MSG_OK;
}

// Per-system device setup (element matrices, E field, load, Jacobi diagonal),
// the system table (fields a caller set before, z, rl and lmap, are kept), the
// work items and the scalars' layout on the device.
static int rg_batch_upload(Context* ctx, const std::vector<RgInput>& in, RgBatch& b) {
  cudaStream_t st = ctx->stream;
  for (int i = 0; i < b.S; ++i) {
    RgBuf& B = b.bufs[i];
    MSG_TRY(rg_setup(ctx, in[i], B, b.k300, b.d_status));
    Mesh* m = in[i].m;
    RgSys& Y = b.sys[i];
    Y.n_nodes = m->n_nodes;
    Y.Rp = B.Rp;
    Y.n_blk = B.n_blk;
    Y.n_blk_u = B.n_blk_u;
    Y.inc_ptr = B.ptr;
    Y.inc = B.inc;
    Y.conn = m->d_conn.as<int>();
    Y.mask = m->d_mask.as<uint8_t>();
    Y.K32 = B.K32;
    Y.K64 = B.K64;
    Y.E32 = B.E32;
    Y.E64 = B.E64;
    Y.b = B.bn;
    Y.x = B.x;
    Y.d = B.d;
    Y.r = B.r;
    Y.p = B.p;
    Y.q = B.q;
    Y.dinv = B.dinv;
    Y.part = B.part;
    Y.part_u = B.part_u;
    if (b.z[i]) Y.z = b.z[i];
  }
  MSG_CUDA(ctx, cudaMemcpyAsync(b.d_sys, b.sys.data(), sizeof(RgSys) * b.S, cudaMemcpyHostToDevice, st));
  MSG_CUDA(ctx, cudaMemcpyAsync(b.d_items, b.items.data(), sizeof(RgItem) * b.items.size(), cudaMemcpyHostToDevice,
                                st));
  MSG_CUDA(ctx, cudaMemcpyAsync(b.d_items_u, b.items_u.data(), sizeof(RgItem) * b.items_u.size(),
                                cudaMemcpyHostToDevice, st));
  const int Rtot = b.Rtot;
  RgScal& s = b.s;
  s.gamma = reinterpret_cast<double*>(b.scal_base);
  s.rr_ref = s.gamma + Rtot;
  s.bnorm = s.rr_ref + Rtot;
  s.res = s.bnorm + Rtot;
  s.alpha = reinterpret_cast<float*>(s.res + Rtot);
  s.beta = s.alpha + Rtot;
  s.done = reinterpret_cast<int*>(s.beta + Rtot);
  s.its = s.done + Rtot;
  s.rsys = s.its + Rtot;
  s.sreq = s.rsys + Rtot;
  s.gact = s.sreq + b.S;
  s.flags = s.gact + Rtot / 32;
  MSG_CUDA(ctx, cudaMemcpyAsync(s.rsys, b.rsys.data(), sizeof(int) * Rtot, cudaMemcpyHostToDevice, st));
  MSG_CUDA(ctx, cudaMemsetAsync(s.sreq, 0, sizeof(int) * b.S, st));
  return MSG_OK;
}

int ebe_ragged_solve(Context* ctx, const std::vector<RgInput>& in, int max_it, double tol) {
  NvtxRange range("msg: batched element-by-element solve");
  if (in.empty() || max_it <= 0 || !(tol > 0))
    return set_error(ctx, MSG_ERR_INVALID_ARGUMENT, "element-by-element batch: invalid arguments");
  cudaStream_t st = ctx->stream;
  const auto t_setup = std::chrono::steady_clock::now();
  const int S = (int)in.size();
  RgBatch b;
  MSG_TRY(rg_batch_plan(ctx, in, std::vector<int>(S, 32), std::vector<int>(S, 0), b));
  MSG_TRY(rg_batch_upload(ctx, in, b));
  const std::vector<RgBuf>& bufs = b.bufs;
  const std::vector<RgSys>& sys = b.sys;
  const int Rtot = b.Rtot, n_items = b.n_items, n_items_u = b.n_items_u;
  const RgScal s = b.s;
  for (int i = 0; i < S; ++i) {
    const dim3 g(bufs[i].n_blk, bufs[i].Rp / 32);
    k_rg_init<<<g, 32 * kEbeWarps, 0, st>>>(sys[i]);
    k_rg_start<<<bufs[i].Rp / kEbeWarps, 32 * kEbeWarps, 0, st>>>(sys[i], in[i].R, s);
    count_launch(ctx, 2);
  }
  const int n_groups = Rtot / 32, g_groups = (n_groups + kEbeWarps - 1) / kEbeWarps;
  k_rg_active<<<g_groups, 32 * kEbeWarps, 0, st>>>(n_groups, s);
  count_launch(ctx);
  MSG_CUDA(ctx, cudaGetLastError());
  // persistent grids: the CTAs that fit on the device at once, at most one per item
  int occ_apply = 1, occ_update = 1, occ_resid = 1;
  MSG_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_apply, k_rg_apply, 32 * kEbeWarps, 0));
  MSG_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_update, k_rg_update, 32 * kEbeWarps, 0));
  MSG_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_resid, k_rg_resid64, 32 * kEbeWarps, 0));
  auto grid_of = [&](int occ, int n) { return std::max(1, std::min(n, ctx->sm_count * std::max(1, occ))); };
  const int g_apply = grid_of(occ_apply, n_items), g_update = n_items_u;
  const int g_resid = grid_of(occ_resid, n_items), g_fold = grid_of(occ_update, n_items);
  const int g_scal = (Rtot + kEbeWarps - 1) / kEbeWarps;
  const RgSys* dS = b.d_sys;
  const RgItem* dI = b.d_items;
  const RgItem* dIu = b.d_items_u;
  const double delta2 = ctx->reliable_delta * ctx->reliable_delta, tol2 = 0.25 * tol * tol;
  // one chunk of kEbeCheck iterations, captured once as a CUDA graph
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  MSG_CUDA(ctx, cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
  cudaMemsetAsync(s.flags, 0, 2 * sizeof(int), st);
  for (int k = 0; k < kEbeCheck; ++k) {
    k_rg_apply<<<g_apply, 32 * kEbeWarps, 0, st>>>(dS, dI, n_items, s.gact, 0);
    k_rg_scalar<<<g_scal, 32 * kEbeWarps, 0, st>>>(dS, Rtot, s, k > 0, tol2, delta2, max_it);
    k_rg_update<<<g_update, 32 * kEbeWarps, 0, st>>>(dS, dIu, n_items_u, s);
  }
  k_rg_chunk_end<<<g_scal, 32 * kEbeWarps, 0, st>>>(dS, Rtot, s, tol2, delta2, max_it);
  const cudaError_t ce = cudaStreamEndCapture(st, &graph);
  if (ce != cudaSuccess) return cuda_error(ctx, ce, "cudaStreamEndCapture");
  const cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
  cudaGraphDestroy(graph);
  if (ie != cudaSuccess) return cuda_error(ctx, ie, "cudaGraphInstantiate");
  struct ExecGuard {
    cudaGraphExec_t e;
    ~ExecGuard() { cudaGraphExecDestroy(e); }
  } guard{exec};
  int* h = ctx->h_flags;
  int n_true = 0;
  MSG_CUDA(ctx, cudaStreamSynchronize(st));
  ctx->t_phase[0] = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_setup).count();
  cudaEventRecord(ctx->ev[10], st);
  // a chunk adds kEbeCheck products to every running realization and one at
  // the limit asks for a true residual, which stops it: the loop ends after at
  // most max_it / kEbeCheck + 1 chunks
  const int max_chunks = max_it / kEbeCheck + 2;
  for (int chunk = 0; chunk < max_chunks; ++chunk) {
    MSG_CUDA(ctx, cudaGraphLaunch(exec, st));
    count_launch(ctx, 3 * kEbeCheck + 1);
    MSG_TRY(publish_flags(ctx, s.flags, 2, h, ctx->d_hflags, st));
    MSG_CUDA(ctx, cudaStreamSynchronize(st));
    if (h[1] == 0) break;
    if (h[0] == 0) continue;
    ++n_true;
    MSG_CUDA(ctx, cudaMemsetAsync(s.flags + 1, 0, sizeof(int), st));
    k_rg_fold<<<g_fold, 32 * kEbeWarps, 0, st>>>(dS, dI, n_items, s, 0);
    k_rg_resid64<<<g_resid, 32 * kEbeWarps, 0, st>>>(dS, dI, n_items, s);
    k_rg_true<<<g_scal, 32 * kEbeWarps, 0, st>>>(dS, Rtot, s, tol, max_it);
    k_rg_active<<<g_groups, 32 * kEbeWarps, 0, st>>>(n_groups, s);
    MSG_CUDA(ctx, cudaMemsetAsync(s.sreq, 0, sizeof(int) * S, st));
    count_launch(ctx, 4);
    MSG_CUDA(ctx, cudaGetLastError());
    MSG_TRY(publish_flags(ctx, s.flags + 1, 1, h + 1, ctx->d_hflags ? ctx->d_hflags + 1 : nullptr, st));
    MSG_CUDA(ctx, cudaStreamSynchronize(st));
    if (h[1] == 0) break;
  }
  cudaEventRecord(ctx->ev[11], st);
  MSG_CUDA(ctx, cudaEventSynchronize(ctx->ev[11]));
  float loop_ms = 0.f;
  cudaEventElapsedTime(&loop_ms, ctx->ev[10], ctx->ev[11]);
  ctx->t_phase[1] = loop_ms;
  ctx->t_phase[2] = n_true;
  ctx->t_phase[3] = 0.0;
  // results (a realization stops right after its fold, so this adds 0 to it
  // unless it broke down or the chunk bound ended the loop)
  k_rg_fold<<<g_fold, 32 * kEbeWarps, 0, st>>>(dS, dI, n_items, s, 1);
  count_launch(ctx);
  return rg_results(ctx, in, bufs, sys, s, Rtot);
}

int ebe_mg_solve(Context* ctx, const std::vector<RgInput>& in, const std::vector<int>& use_vcycle, int max_it,
                 double tol) {
  NvtxRange range("msg: preconditioned element-by-element solve");
  if (in.empty() || in.size() != use_vcycle.size() || max_it <= 0 || !(tol > 0))
    return set_error(ctx, MSG_ERR_INVALID_ARGUMENT, "element-by-element batch: invalid arguments");
  cudaStream_t st = ctx->stream;
  const auto t_setup = std::chrono::steady_clock::now();
  const int S = (int)in.size();
  if (S > 1000) return set_error(ctx, MSG_ERR_INVALID_ARGUMENT, "element-by-element batch: more than 1000 systems");
  std::vector<Mesh*> lats(S, nullptr);
  std::vector<int> rp_multiple(S), want_z(S);
  for (int i = 0; i < S; ++i) {
    if (!in[i].m || in[i].m->ctx != ctx)
      return set_error(ctx, MSG_ERR_INVALID_ARGUMENT, "element-by-element batch: system %d has no mesh of this context", i);
    if (use_vcycle[i]) MSG_TRY(lattice_shadow(ctx, in[i].m, &lats[i]));
    // the packed level-0 operator of a V-cycle takes pairs of realization groups;
    // z of a V-cycle system is the lattice's own buffer
    rp_multiple[i] = use_vcycle[i] ? 64 : 32;
    want_z[i] = use_vcycle[i] ? 0 : 1;
  }
  RgBatch b;
  MSG_TRY(rg_batch_plan(ctx, in, rp_multiple, want_z, b));
  const std::vector<RgBuf>& bufs = b.bufs;
  // preconditioners: the V-cycle of each system's cube lattice (lattice buffers
  // of their own when several systems hold one), E of every realization on the
  // lattice's elements; r and z of such a system live in the lattice's buffers
  int n_vc = 0;
  for (int i = 0; i < S; ++i) n_vc += use_vcycle[i] ? 1 : 0;
  std::vector<void*> P(S, nullptr);
  struct PGuard {
    std::vector<void*>& p;
    ~PGuard() {
      for (void* q : p)
        if (q) gmg_precond_destroy(q);
    }
  } pguard{P};
  if (n_vc > 1)
    while ((int)ctx->vc_pool.size() < n_vc) ctx->vc_pool.push_back(new DevMem[kWorkSlots]);
  for (int i = 0, k = 0; i < S; ++i) {
    b.sys[i].kind = use_vcycle[i] ? 1 : 0;
    if (!use_vcycle[i]) continue;
    DevMem* own = n_vc > 1 ? ctx->vc_pool[k++] : nullptr;
    MSG_TRY(gmg_precond_create(ctx, lats[i], in[i].nu, in[i].kl, in[i].d_xi, in[i].R, bufs[i].Rp, own, &P[i]));
    float *rl = nullptr, *zl = nullptr;
    const int* lmap = nullptr;
    const double* lzr = nullptr;
    int lrp = 0, lzr_blocks = 0;
    gmg_precond_buffers(P[i], &rl, &zl, &lmap, &lrp, &lzr, &lzr_blocks);
    if (lrp != bufs[i].Rp)
      return set_error(ctx, MSG_ERR_UNKNOWN, "element-by-element batch: lattice layout of %d realizations, not %d",
                       lrp, bufs[i].Rp);
    b.sys[i].rl = rl;
    b.sys[i].z = zl;
    b.sys[i].lmap = lmap;
    b.sys[i].lzr = lzr;
    b.sys[i].lzr_blocks = lzr_blocks;
  }
  MSG_TRY(rg_batch_upload(ctx, in, b));
  const std::vector<RgSys>& sys = b.sys;
  const int Rtot = b.Rtot, n_items = b.n_items, n_items_u = b.n_items_u;
  const RgScal s = b.s;
  const RgItem* d_items = b.d_items;
  const RgItem* d_items_u = b.d_items_u;
  const RgSys* dS = b.d_sys;
  const int n_groups = Rtot / 32, g_groups = (n_groups + kEbeWarps - 1) / kEbeWarps;
  const int g_scal = (Rtot + kEbeWarps - 1) / kEbeWarps;
  int occ_apply = 1, occ_resid = 1, occ_u = 1;
  MSG_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_apply, k_rg_apply, 32 * kEbeWarps, 0));
  MSG_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_resid, k_rg_resid64, 32 * kEbeWarps, 0));
  MSG_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_u, k_rg_fold, 32 * kEbeWarps, 0));
  auto grid_of = [&](int occ, int n) { return std::max(1, std::min(n, ctx->sm_count * std::max(1, occ))); };
  const int g_apply = grid_of(occ_apply, n_items), g_resid = grid_of(occ_resid, n_items);
  const int g_fold = grid_of(occ_u, n_items), g_u = n_items_u;
  // z = M^-1 r of the systems in `which` (nullptr: all): V-cycles one system
  // after another, the diagonal for all the others in one launch. from_node:
  // r of the V-cycle systems in node layout (the start and the true
  // residuals); in the loop the update pass has written it to the lattice
  auto precondition = [&](const std::vector<int>* which, bool from_node) -> int {
    for (int i = 0; i < S; ++i)
      if (P[i] && (!which || (*which)[i]))
        MSG_TRY(gmg_precond_apply(ctx, P[i], from_node ? bufs[i].r : nullptr, nullptr, st));
    if (n_vc < S) {
      k_vc_jacobi_z<<<g_u, 32 * kEbeWarps, 0, st>>>(dS, d_items_u, n_items_u, s);
      count_launch(ctx);
    }
    return MSG_OK;
  };
  // start: x = 0, d = 0, r = b, ||b||; z = M^-1 b, gamma = z.b, p = z
  for (int i = 0; i < S; ++i) {
    k_rg_init<<<dim3(bufs[i].n_blk, bufs[i].Rp / 32), 32 * kEbeWarps, 0, st>>>(sys[i]);
    count_launch(ctx);
  }
  MSG_CUDA(ctx, cudaMemsetAsync(s.gact, 0xff, sizeof(int) * n_groups, st));  // every group until the start
  MSG_TRY(precondition(nullptr, true));
  for (int i = 0; i < S; ++i) k_vc_start<<<bufs[i].Rp / kEbeWarps, 32 * kEbeWarps, 0, st>>>(sys[i], in[i].R, s);
  k_rg_active<<<g_groups, 32 * kEbeWarps, 0, st>>>(n_groups, s);
  k_vc_dir<<<g_u, 32 * kEbeWarps, 0, st>>>(dS, d_items_u, n_items_u, s);
  count_launch(ctx, 2 + S);
  MSG_CUDA(ctx, cudaGetLastError());
  // two iterations to a graph launch (the multigrid loop's chunk), its reliable-update factor
  constexpr int kChunk = 2;
  const double delta2 = ctx->mg_delta * ctx->mg_delta, tol2 = 0.25 * tol * tol;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  MSG_CUDA(ctx, cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
  cudaMemsetAsync(s.flags, 0, 2 * sizeof(int), st);
  for (int k = 0; k < kChunk; ++k) {
    k_rg_apply<<<g_apply, 32 * kEbeWarps, 0, st>>>(dS, d_items, n_items, s.gact, 1);
    k_vc_alpha<<<g_scal, 32 * kEbeWarps, 0, st>>>(dS, Rtot, s);
    k_vc_update<<<g_u, 32 * kEbeWarps, 0, st>>>(dS, d_items_u, n_items_u, s);
    precondition(nullptr, false);
    k_vc_beta<<<g_scal, 32 * kEbeWarps, 0, st>>>(dS, Rtot, s, tol2, delta2, max_it);
    k_vc_dir<<<g_u, 32 * kEbeWarps, 0, st>>>(dS, d_items_u, n_items_u, s);
  }
  k_rg_chunk_end_count<<<g_scal, 32 * kEbeWarps, 0, st>>>(Rtot, s);
  const cudaError_t ce = cudaStreamEndCapture(st, &graph);
  if (ce != cudaSuccess) return cuda_error(ctx, ce, "cudaStreamEndCapture");
  const cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
  cudaGraphDestroy(graph);
  if (ie != cudaSuccess) return cuda_error(ctx, ie, "cudaGraphInstantiate");
  struct ExecGuard {
    cudaGraphExec_t e;
    ~ExecGuard() { cudaGraphExecDestroy(e); }
  } guard{exec};
  int* h = ctx->h_flags;
  int* hreq = ctx->h_flags + 16;  // per-system requests (mapped words 16 .. 16 + S)
  int n_true = 0;
  std::vector<int> req(S, 0);
  MSG_CUDA(ctx, cudaStreamSynchronize(st));
  ctx->t_phase[0] = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_setup).count();
  cudaEventRecord(ctx->ev[10], st);
  const int max_chunks = max_it / kChunk + 2;
  for (int chunk = 0; chunk < max_chunks; ++chunk) {
    MSG_CUDA(ctx, cudaGraphLaunch(exec, st));
    count_launch(ctx, kChunk * (5 + n_vc + (n_vc < S ? 1 : 0)) + 1);
    MSG_TRY(publish_flags(ctx, s.flags, 2, h, ctx->d_hflags, st));
    MSG_CUDA(ctx, cudaStreamSynchronize(st));
    if (h[1] == 0) break;
    if (h[0] == 0) continue;
    // the systems that asked: FP64 true residual, z = M^-1 r, gamma = z.r; each
    // of their running realizations stops or continues
    ++n_true;
    MSG_TRY(publish_flags(ctx, s.sreq, S, hreq, ctx->d_hflags ? ctx->d_hflags + 16 : nullptr, st));
    MSG_CUDA(ctx, cudaStreamSynchronize(st));
    for (int i = 0; i < S; ++i) req[i] = hreq[i];
    MSG_CUDA(ctx, cudaMemsetAsync(s.flags + 1, 0, sizeof(int), st));
    k_rg_fold<<<g_fold, 32 * kEbeWarps, 0, st>>>(dS, d_items, n_items, s, 0);
    k_rg_resid64<<<g_resid, 32 * kEbeWarps, 0, st>>>(dS, d_items, n_items, s);
    MSG_TRY(precondition(&req, true));
    k_vc_true<<<g_scal, 32 * kEbeWarps, 0, st>>>(dS, Rtot, s, tol, max_it);
    k_rg_active<<<g_groups, 32 * kEbeWarps, 0, st>>>(n_groups, s);
    MSG_CUDA(ctx, cudaMemsetAsync(s.sreq, 0, sizeof(int) * S, st));
    count_launch(ctx, 4);
    MSG_CUDA(ctx, cudaGetLastError());
    MSG_TRY(publish_flags(ctx, s.flags + 1, 1, h + 1, ctx->d_hflags ? ctx->d_hflags + 1 : nullptr, st));
    MSG_CUDA(ctx, cudaStreamSynchronize(st));
    if (h[1] == 0) break;
  }
  cudaEventRecord(ctx->ev[11], st);
  MSG_CUDA(ctx, cudaEventSynchronize(ctx->ev[11]));
  float loop_ms = 0.f;
  cudaEventElapsedTime(&loop_ms, ctx->ev[10], ctx->ev[11]);
  ctx->t_phase[1] = loop_ms;
  ctx->t_phase[2] = n_true;
  ctx->t_phase[3] = 0.0;
  k_rg_fold<<<g_fold, 32 * kEbeWarps, 0, st>>>(dS, d_items, n_items, s, 1);
  count_launch(ctx);
  return rg_results(ctx, in, bufs, sys, s, Rtot);
}

int ebe_solve(Context* ctx, const std::vector<RgInput>& in, int max_it, double tol) {
  std::vector<int> vc(in.size(), 0);
  bool any = false;
  for (size_t i = 0; i < in.size(); ++i) {
    const Mesh* m = in[i].m;
    if (!m || ctx->multigrid == 0 || ctx->mg_levels < 2) continue;
    const int nx = m->structured ? m->nx : m->tnx, ny = m->structured ? m->ny : m->tny,
              nz = m->structured ? m->nz : m->tnz;
    const bool lattice = m->structured || m->topo_lattice;
    vc[i] = lattice && nx % 2 == 0 && ny % 2 == 0 && nz % 2 == 0 && nx >= 4 && ny >= 4 && nz >= 4;
    any = any || vc[i];
  }
  // the loop publishes one request word a system into the mapped flag page
  return any && in.size() <= 1000 ? ebe_mg_solve(ctx, in, vc, max_it, tol) : ebe_ragged_solve(ctx, in, max_it, tol);
}

}  // namespace msg
