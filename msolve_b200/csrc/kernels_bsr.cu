// Assembled FP64 path: 3x3 block sliced-ELL (SELL-32) stiffness built on the
// device from element matrices, its SpMV, and a Jacobi-PCG whose whole loop
// runs on the device.
//
// Replaces the skyline assembler (GlobalMatrixAssemblerSkyline.cs:51-103), the
// skyline product (SkylineMatrix2D.Multiply :224-286) and the PCG loop of
// SolverPCG.Solve (PCG/SolverPCG.cs:105-149) with the simple search vector
// (SolverPCGSimpleSearchVectorCalculator.cs:18-41) and the diagonal
// preconditioner z_j = r_j / K_jj (PolynomialChaosSolverPCGMatrixCalculator.cs:467-495).
//
// Layout: block row = mesh node; vectors in node layout v[3*node + comp]
// (constrained components hold 0 and their matrix rows/columns are identity).
// SELL values: val[((slot)*9 + k)*32 + lane], k = 3*row_comp + col_comp, so a
// warp reads each of the 9 block entries of 32 consecutive rows as one 256-byte
// coalesced load; the matrix stream is the whole HBM traffic of the product.
#include <algorithm>

#include <cstddef>

#include "msg_internal.h"

namespace msg {
namespace {


// One thread per (flat position, block entry k): sum the element
// contributions (e, a, b) of this block in their fixed order, then apply the
// Dirichlet mask (identity on constrained rows/columns).
__global__ void k_bsr_assemble(int64_t n_pos, const int* __restrict__ /*col*/, const int64_t* __restrict__ cptr,
                               const int* __restrict__ contrib, const double* __restrict__ Ke,
                               double* __restrict__ val) {
  const int64_t tid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (tid >= n_pos * 9) return;
  const int64_t pos = tid / 9;
  const int k = (int)(tid - pos * 9);
  const int64_t slot = pos >> 5;
  const int lane = (int)(pos & 31);
  const int cr = k / 3, cc = k - 3 * cr;
  double acc = 0.0;
  for (int64_t q = cptr[pos]; q < cptr[pos + 1]; ++q) {
    const int code = contrib[q];
    const int e = code >> 6, a = (code >> 3) & 7, b = code & 7;
    acc += Ke[(size_t)e * 300 + packed_index(3 * a + cr, 3 * b + cc)];
  }
  val[(slot * 9 + k) * 32 + lane] = acc;
}

// Dirichlet masking pass: row node = slice*32 + lane, column node = col[pos].
__global__ void k_bsr_mask(int n_rows, const int64_t* __restrict__ slice_ptr, const int* __restrict__ col,
                           const uint8_t* __restrict__ mask, double* __restrict__ val) {
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= n_rows) return;
  const int slice = row >> 5, lane = row & 31;
  const int64_t s0 = slice_ptr[slice], s1 = slice_ptr[slice + 1];
  const uint8_t mr = mask[row];
  for (int64_t s = s0; s < s1; ++s) {
    const int c = col[s * 32 + lane];
    if (c < 0) break;
    const uint8_t mc = mask[c];
    if ((mr | mc) == 0) continue;
#pragma unroll
    for (int k = 0; k < 9; ++k) {
      const int cr = k / 3, cc = k % 3;
      if (((mr >> cr) & 1) || ((mc >> cc) & 1)) val[(s * 9 + k) * 32 + lane] = (c == row && cr == cc) ? 1.0 : 0.0;
    }
  }
}

__global__ void k_bsr_diag_inv(int n_rows, const int* __restrict__ diag_pos, const double* __restrict__ val,
                               double* __restrict__ dinv) {
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= n_rows) return;
  const int64_t pos = diag_pos[row];
  const int64_t slot = pos >> 5;
  const int lane = (int)(pos & 31);
#pragma unroll
  for (int c = 0; c < 3; ++c) dinv[3 * row + c] = 1.0 / val[(slot * 9 + 4 * c) * 32 + lane];
}

// One warp per (32-row slice, output component): 3x the threads of a
// row-per-thread product, each warp still reading its 3 block entries per
// slot as coalesced 256-byte lines.
__device__ __forceinline__ double sell_row_comp(int slice, int lane, int c, const int64_t* __restrict__ slice_ptr,
                                                const int* __restrict__ col, const double* __restrict__ val,
                                                const double* __restrict__ x) {
  const int64_t s0 = slice_ptr[slice], s1 = slice_ptr[slice + 1];
  double acc = 0;
  for (int64_t s = s0; s < s1; ++s) {
    const int cc = __ldg(col + s * 32 + lane);
    if (cc < 0) break;
    const double* v = val + (s * 9 + 3 * c) * 32 + lane;
    acc += __ldg(v) * __ldg(x + 3 * cc) + __ldg(v + 32) * __ldg(x + 3 * cc + 1) + __ldg(v + 64) * __ldg(x + 3 * cc + 2);
  }
  return acc;
}

__global__ void __launch_bounds__(96) k_bsr_spmv3(int n_rows, const int64_t* __restrict__ slice_ptr,
                                                  const int* __restrict__ col, const double* __restrict__ val,
                                                  const double* __restrict__ x, double* __restrict__ y) {
  const int slice = blockIdx.x, c = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int row = slice * 32 + lane;
  if (row >= n_rows) return;
  y[3 * row + c] = sell_row_comp(slice, lane, c, slice_ptr, col, val, x);
}

__global__ void k_dof_to_node(int n_dofs, const int* __restrict__ free_rows, const double* __restrict__ in,
                              double* __restrict__ out, int64_t in_stride, int64_t out_stride) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int v = blockIdx.y;
  if (i >= n_dofs) return;
  out[v * out_stride + free_rows[i]] = in[v * in_stride + i];
}

__global__ void k_node_to_dof(int n_dofs, const int* __restrict__ free_rows, const double* __restrict__ in,
                              double* __restrict__ out, int64_t in_stride, int64_t out_stride) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int v = blockIdx.y;
  if (i >= n_dofs) return;
  out[v * out_stride + i] = in[v * in_stride + free_rows[i]];
}

// ------------------------------------------------------------------ PCG
// Device-resident Jacobi-PCG. Two kernels per iteration, each ending with a
// last-block-done reduction that updates the scalar state in fixed block order
// (deterministic results):
//   k_pcg_dir_spmv: p_new = dinv.r + beta p_old (recomputed for gathered
//     columns, written for own rows), q = K p_new, partial p.q
//     -> last block: alpha = z.r / p.q (breakdown check)
//   k_pcg_update:   r -= alpha q, x += alpha p_new, partials r.r and (dinv r).r
//     -> last block: err = ||r||/||b||, convergence / iteration bookkeeping, beta
// p is double-buffered by iteration parity so gathered columns are never read
// while being overwritten.

constexpr int kPcgThreads = 256;

__device__ __forceinline__ double block_sum(double v, double* sh) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) sh[w] = v;
  __syncthreads();
  double s = 0;
  if (threadIdx.x == 0)
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) s += sh[i];
  return s;  // valid in thread 0
}

// Whole-block sums of the K interleaved partials partial[i*K + k], i < n, in a
// fixed order (thread t adds i = t, t + blockDim, ... in turn; then the block
// tree): called by every thread of the last block, results valid in thread 0.
// The loads of four rounds are issued before their adds (the order of the adds
// is unchanged), so the last block waits for one L2 round trip, not n / blockDim.
template <int K>
__device__ __forceinline__ void sum_partials(const double* partial, int n, double (&out)[K], double* sh) {
  double s[K];
#pragma unroll
  for (int k = 0; k < K; ++k) s[k] = 0;
  const int B = blockDim.x;
  int i = threadIdx.x;
  for (; i + 3 * B < n; i += 4 * B) {
    double v[4][K];
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
      for (int k = 0; k < K; ++k) v[u][k] = __ldcg(partial + (size_t)(i + u * B) * K + k);
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
      for (int k = 0; k < K; ++k) s[k] += v[u][k];
  }
  for (; i < n; i += B)
#pragma unroll
    for (int k = 0; k < K; ++k) s[k] += __ldcg(partial + (size_t)i * K + k);
#pragma unroll
  for (int k = 0; k < K; ++k) out[k] = block_sum(s[k], sh);
}

// Returns true in every thread of the last block to finish.
__device__ __forceinline__ bool last_block(unsigned int* counter) {
  __shared__ bool is_last;
  __threadfence();
  if (threadIdx.x == 0) {
    const unsigned int ticket = atomicAdd(counter, 1u);
    is_last = (ticket == gridDim.x - 1);
  }
  __syncthreads();
  return is_last;
}

__global__ void __launch_bounds__(kPcgThreads) k_pcg_init(int n_rows, const double* __restrict__ b,
                                                          const double* __restrict__ dinv, double* __restrict__ r,
                                                          double* __restrict__ x, double* __restrict__ p0,
                                                          double* __restrict__ p1, double* __restrict__ partial,
                                                          PcgState* st) {
  __shared__ double sh[32];
  double bb = 0, zr = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < 3 * n_rows; i += gridDim.x * blockDim.x) {
    const double bi = b[i];
    r[i] = bi; x[i] = 0; p0[i] = 0; p1[i] = 0;
    bb += bi * bi;
    zr += bi * dinv[i] * bi;
  }
  double s1 = block_sum(bb, sh);
  double s2 = block_sum(zr, sh);
  if (threadIdx.x == 0) { partial[2 * blockIdx.x] = s1; partial[2 * blockIdx.x + 1] = s2; }
  if (!last_block(&st->counter)) return;
  double tt[2];
  sum_partials<2>(partial, gridDim.x, tt, sh);
  const double tb = tt[0], tz = tt[1];
  if (threadIdx.x == 0) {
    st->bnorm = sqrt(tb);
    st->zr = tz;
    st->beta = 0; st->alpha = 0; st->err = 0;
    st->it = 0; st->iterations = 0; st->matvecs = 0; st->status = 0;
    st->done = (st->bnorm > 1e-25) ? 0 : 1;  // SolverPCG.cs:112
    st->need = 0; st->err_ref = 1.0;
    st->counter = 0;
  }
}

// The loop's direction + SpMV kernel: p_new = dinv.r + beta p_old (formed for
// gathered columns, written for own rows), q = K p_new, partial p.q -> last
// block: alpha = z.r / p.q (breakdown check). A CTA is one 32-row slice, a
// thread owns the 3 components of its row, so every slot streams 9 coalesced
// 256-byte value lines per warp and the gathered p is formed once per column
// (not once per output component). A CTA takes kS slices; a slice's slots are
// dealt round-robin to kW warps (kW = 4 for small matrices, to keep enough
// warps in flight; 1 for large ones) and the warp sums meet in shared memory
// in fixed order. Slots are taken in groups
// whose value loads are all issued before use (144 bytes in flight per
// thread); values of matrices too large for L2 stream with evict-first loads
// so the vectors stay in L2 (smaller ones stay in L2 across iterations);
// padded positions (column -1) hold zero values and skip the gather.
template <class V, int kS, int kSpmvWarps, bool kStream>
__global__ void __launch_bounds__(32 * kS * kSpmvWarps) k_pcg_dir_spmv_rows(int n_rows, int n_slices,
                                                                      const int64_t* __restrict__ slice_ptr,
                                                                      const int* __restrict__ col,
                                                                      const V* __restrict__ val,
                                                                      const double* __restrict__ dinv,
                                                                      const double* __restrict__ r, double* p0,
                                                                      double* p1, double* __restrict__ q,
                                                                      double* __restrict__ partial, PcgState* st) {
  __shared__ double sh[32];
  __shared__ double ys[kS][kSpmvWarps][3][32];
  if (st->done) return;
  const int it = st->it;
  const double beta = st->beta;
  const double* __restrict__ pold = (it & 1) ? p1 : p0;
  double* __restrict__ pnew = (it & 1) ? p0 : p1;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int sl = warp / kSpmvWarps, w = warp % kSpmvWarps;
  const int slice = blockIdx.x * kS + sl;
  const int row = slice * 32 + lane;
  const bool live = slice < n_slices && row < n_rows;
  double y0 = 0, y1 = 0, y2 = 0;
  auto fma9 = [&](const double (&a)[9], int cc) {
    if (cc < 0) return;  // padding (its values are zero)
    const double x0 = dinv[3 * cc] * r[3 * cc] + beta * pold[3 * cc];
    const double x1 = dinv[3 * cc + 1] * r[3 * cc + 1] + beta * pold[3 * cc + 1];
    const double x2 = dinv[3 * cc + 2] * r[3 * cc + 2] + beta * pold[3 * cc + 2];
    y0 += a[0] * x0 + a[1] * x1 + a[2] * x2;
    y1 += a[3] * x0 + a[4] * x1 + a[5] * x2;
    y2 += a[6] * x0 + a[7] * x1 + a[8] * x2;
  };
  if (live) {
    const int64_t s0 = slice_ptr[slice], s1 = slice_ptr[slice + 1];
    constexpr int U = 16 / (int)sizeof(V);  // 2 FP64 / 4 FP32 slots per group
    int64_t s = s0 + w;
    for (; s + (U - 1) * kSpmvWarps < s1; s += U * kSpmvWarps) {
      int cu[U];
      double a[U][9];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int64_t su = s + u * kSpmvWarps;
        cu[u] = __ldg(col + su * 32 + lane);
        const V* vu = val + su * 9 * 32 + lane;
#pragma unroll
        for (int k = 0; k < 9; ++k) a[u][k] = (double)(kStream ? __ldcs(vu + k * 32) : __ldg(vu + k * 32));
      }
#pragma unroll
      for (int u = 0; u < U; ++u) fma9(a[u], cu[u]);
    }
    for (; s < s1; s += kSpmvWarps) {
      const int c0 = __ldg(col + s * 32 + lane);
      const V* v0 = val + s * 9 * 32 + lane;
      double a0[9];
#pragma unroll
      for (int k = 0; k < 9; ++k) a0[k] = (double)(kStream ? __ldcs(v0 + k * 32) : __ldg(v0 + k * 32));
      fma9(a0, c0);
    }
  }
  ys[sl][w][0][lane] = y0;
  ys[sl][w][1][lane] = y1;
  ys[sl][w][2][lane] = y2;
  __syncthreads();
  double pq = 0;
  if (w == 0 && live) {
    double yc[3], pn[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      double t = ys[sl][0][c][lane];
#pragma unroll
      for (int ww = 1; ww < kSpmvWarps; ++ww) t += ys[sl][ww][c][lane];
      yc[c] = t;
      pn[c] = dinv[3 * row + c] * r[3 * row + c] + beta * pold[3 * row + c];
      pnew[3 * row + c] = pn[c];
      q[3 * row + c] = t;
    }
    pq = pn[0] * yc[0] + pn[1] * yc[1] + pn[2] * yc[2];
  }
  const double bs = block_sum(pq, sh);
  if (threadIdx.x == 0) partial[blockIdx.x] = bs;
  if (!last_block(&st->counter)) return;
  double tt[1];
  sum_partials<1>(partial, gridDim.x, tt, sh);
  const double t = tt[0];
  if (threadIdx.x == 0) {
    st->pq = t;
    st->matvecs += 1;
    if (!(t > 0) || isnan(t)) {  // breakdown: p.q <= 0 or NaN
      st->status = MSG_ERR_BREAKDOWN; st->done = 1; st->iterations = it;
    } else {
      st->alpha = st->zr / t;
    }
    st->counter = 0;
  }
}

// ------------------------------------------------------------------ mixed-precision PCG
// MSG_PCG_SOLVE_MIXED's loop: FP32 matrix values and FP32 vectors (r, p, q, the
// correction d and D^-1) inside the loop, the iterate x in FP64 (x += d at each
// FP64 true residual) and FP64 sums for every dot product. Two kernels an
// iteration:
//   k_pcgm_spmv:   q = K32 p (p gathered in FP32), partials p.q, (D r).q and
//     q.D q -> last block: alpha = gamma / p.q (breakdown check) and, since
//     r' = r - alpha q, gamma' = (D r').r' = gamma - 2 alpha (D r).q +
//     alpha^2 q.D q, hence beta = gamma' / gamma before the update;
//   k_pcgm_update: r -= alpha q, d += alpha p, z = D r, p = z + beta p (the
//     next direction, formed in the same pass) and the exact z.r, r.r ->
//     last block: gamma = z.r, ||r||/||b||, pause for an FP64 true residual
//     when it has dropped by delta since the last one or below tol.
// On a pause the host runs k_pcgm_fold (x += d, d = 0), y = K64 x with the FP64
// values and k_pcgm_true (r = b - y into the FP32 r, gamma = (D r).r; stop
// when ||r||/||b|| < tol in FP64). The direction is kept across the
// replacement. Per iteration the vectors cost 48 bytes a DOF besides the
// matrix (16 in the SpMV pass, 32 in the update; with FP64 vectors and a
// separate direction pass they would cost 108).
// A warp owns one slice at a time; with kSpmvWarps = 1 the CTAs are persistent
// (the grid fills the SMs once) and a warp strides over the slices, summing its
// partials across them; with kSpmvWarps > 1 (small matrices) a CTA takes one
// slice whose slots are dealt to its warps, whose sums meet in shared memory.
template <int kS, int kSpmvWarps, bool kStream, int U = 4>
__global__ void __launch_bounds__(32 * kS * kSpmvWarps, kSpmvWarps > 1 ? 1 : (U > 4 ? 3 : 4)) k_pcgm_spmv(int n_rows, int n_slices,
                                                              const int64_t* __restrict__ slice_ptr,
                                                              const int* __restrict__ col,
                                                              const float* __restrict__ val,
                                                              const float* __restrict__ p32,
                                                              const float* __restrict__ r32,
                                                              const float* __restrict__ dinv32,
                                                              float* __restrict__ q32, double* __restrict__ partial,
                                                              PcgState* st) {
  __shared__ double sh[32];
  __shared__ double ys[kSpmvWarps > 1 ? kS : 1][kSpmvWarps][3][32];
  if (st->done) return;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int sl = warp / kSpmvWarps, w = warp % kSpmvWarps;
  double pq = 0, dq = 0, qdq = 0;
  const int stride = kSpmvWarps > 1 ? n_slices : gridDim.x * kS;
  for (int slice = blockIdx.x * kS + sl; slice < n_slices || (kSpmvWarps > 1 && slice == blockIdx.x * kS + sl);
       slice += stride) {
    const int row = slice * 32 + lane;
    const bool live = slice < n_slices && row < n_rows;
    double y0 = 0, y1 = 0, y2 = 0;
    auto fma9 = [&](const float (&a)[9], int cc) {
      if (cc < 0) return;  // padding (its values are zero)
      const float x0 = __ldg(p32 + 3 * cc), x1 = __ldg(p32 + 3 * cc + 1), x2 = __ldg(p32 + 3 * cc + 2);
      y0 += (double)fmaf(a[2], x2, fmaf(a[1], x1, a[0] * x0));
      y1 += (double)fmaf(a[5], x2, fmaf(a[4], x1, a[3] * x0));
      y2 += (double)fmaf(a[8], x2, fmaf(a[7], x1, a[6] * x0));
    };
    if (live) {
      const int64_t s0 = slice_ptr[slice], s1 = slice_ptr[slice + 1];
      // U slots per group: 36 U bytes of values in flight per thread
      int64_t s = s0 + w;
      for (; s + (U - 1) * kSpmvWarps < s1; s += U * kSpmvWarps) {
        int cu[U];
        float a[U][9];
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const int64_t su = s + u * kSpmvWarps;
          cu[u] = __ldg(col + su * 32 + lane);
          const float* vu = val + su * 9 * 32 + lane;
#pragma unroll
          for (int k = 0; k < 9; ++k) a[u][k] = kStream ? __ldcs(vu + k * 32) : __ldg(vu + k * 32);
        }
#pragma unroll
        for (int u = 0; u < U; ++u) fma9(a[u], cu[u]);
      }
      for (; s < s1; s += kSpmvWarps) {
        const int c0 = __ldg(col + s * 32 + lane);
        const float* v0 = val + s * 9 * 32 + lane;
        float a0[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) a0[k] = kStream ? __ldcs(v0 + k * 32) : __ldg(v0 + k * 32);
        fma9(a0, c0);
      }
    }
    double yc[3] = {y0, y1, y2};
    if constexpr (kSpmvWarps > 1) {
      ys[sl][w][0][lane] = y0;
      ys[sl][w][1][lane] = y1;
      ys[sl][w][2][lane] = y2;
      __syncthreads();
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        double t = ys[sl][0][c][lane];
#pragma unroll
        for (int ww = 1; ww < kSpmvWarps; ++ww) t += ys[sl][ww][c][lane];
        yc[c] = t;
      }
    }
    if (w == 0 && live) {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const int i = 3 * row + c;
        const float qf = (float)yc[c], dv = dinv32[i];
        q32[i] = qf;
        pq += (double)p32[i] * (double)qf;
        dq += (double)(dv * r32[i]) * (double)qf;
        qdq += (double)(dv * qf) * (double)qf;
      }
    }
    if constexpr (kSpmvWarps > 1) break;
  }
  const double b0 = block_sum(pq, sh), b1 = block_sum(dq, sh), b2 = block_sum(qdq, sh);
  if (threadIdx.x == 0) {
    partial[3 * blockIdx.x] = b0;
    partial[3 * blockIdx.x + 1] = b1;
    partial[3 * blockIdx.x + 2] = b2;
  }
  if (!last_block(&st->counter)) return;
  double tt[3];
  sum_partials<3>(partial, gridDim.x, tt, sh);
  const double t = tt[0], tdq = tt[1], tqdq = tt[2];
  if (threadIdx.x == 0) {
    st->pq = t;
    st->matvecs += 1;
    if (!(t > 0) || isnan(t)) {  // breakdown: p.q <= 0 or NaN
      st->status = MSG_ERR_BREAKDOWN; st->done = 1; st->iterations = st->it;
    } else {
      const double al = st->zr / t;
      const double g1 = st->zr - 2.0 * al * tdq + al * al * tqdq;
      st->alpha = al;
      st->beta = g1 > 0.0 ? g1 / st->zr : 0.0;  // a non-positive estimate restarts from z
    }
    st->counter = 0;
  }
}

// The vectors start at 16-byte boundaries: four components a thread at a
// time (float4), the n3 % 4 tail one at a time.
__global__ void __launch_bounds__(kPcgThreads) k_pcgm_update(int n3, const float* __restrict__ dinv32,
                                                             float* __restrict__ r32, float* __restrict__ p32,
                                                             const float* __restrict__ q32, float* __restrict__ d32,
                                                             double* __restrict__ partial, PcgState* st) {
  __shared__ double sh[32];
  if (st->done) return;
  const float al = (float)st->alpha, be = (float)st->beta;
  double zr = 0, rr = 0;
  auto step = [&](float pv, float qv, float rv, float dv, float dd, float& pn, float& rn, float& dn) {
    rn = fmaf(-al, qv, rv);
    const float zv = dv * rn;
    dn = fmaf(al, pv, dd);
    pn = fmaf(be, pv, zv);
    zr += (double)zv * (double)rn;
    rr += (double)rn * (double)rn;
  };
  const int tid = blockIdx.x * blockDim.x + threadIdx.x, nt = gridDim.x * blockDim.x;
  const int n4 = n3 >> 2;
  for (int i = tid; i < n4; i += nt) {
    const float4 p = reinterpret_cast<const float4*>(p32)[i], q = reinterpret_cast<const float4*>(q32)[i];
    const float4 r = reinterpret_cast<const float4*>(r32)[i], dv = reinterpret_cast<const float4*>(dinv32)[i];
    const float4 d = reinterpret_cast<const float4*>(d32)[i];
    float4 pn, rn, dn;
    step(p.x, q.x, r.x, dv.x, d.x, pn.x, rn.x, dn.x);
    step(p.y, q.y, r.y, dv.y, d.y, pn.y, rn.y, dn.y);
    step(p.z, q.z, r.z, dv.z, d.z, pn.z, rn.z, dn.z);
    step(p.w, q.w, r.w, dv.w, d.w, pn.w, rn.w, dn.w);
    reinterpret_cast<float4*>(p32)[i] = pn;
    reinterpret_cast<float4*>(r32)[i] = rn;
    reinterpret_cast<float4*>(d32)[i] = dn;
  }
  for (int i = 4 * n4 + tid; i < n3; i += nt) step(p32[i], q32[i], r32[i], dinv32[i], d32[i], p32[i], r32[i], d32[i]);
  const double s1 = block_sum(rr, sh), s2 = block_sum(zr, sh);
  if (threadIdx.x == 0) { partial[2 * blockIdx.x] = s1; partial[2 * blockIdx.x + 1] = s2; }
  if (!last_block(&st->counter)) return;
  double tt[2];
  sum_partials<2>(partial, gridDim.x, tt, sh);
  const double tr = tt[0], tz = tt[1];
  if (threadIdx.x == 0) {
    const int it = st->it;
    st->err = sqrt(tr) / st->bnorm;
    st->rr = tr;
    st->zr = tz;
    if (st->err < st->tol || st->err < st->delta * st->err_ref) {
      st->need = 1; st->done = 1;  // pause for an FP64 true residual
    } else if (it + 1 >= st->max_it) {
      st->done = 1; st->iterations = st->max_it; st->status = MSG_ERR_NOT_CONVERGED;
    } else {
      st->it = it + 1;
    }
    st->counter = 0;
  }
}

// Start of the mixed loop: x = 0, d = 0, r = (float) b, D^-1 in FP32, p = z =
// D^-1 r, gamma = z.r, ||b|| in FP64.
__global__ void __launch_bounds__(kPcgThreads) k_pcgm_init(int n3, const double* __restrict__ b,
                                                           const double* __restrict__ dinv, double* __restrict__ x,
                                                           float* __restrict__ r32, float* __restrict__ p32,
                                                           float* __restrict__ d32, float* __restrict__ dinv32,
                                                           double* __restrict__ partial, PcgState* st) {
  __shared__ double sh[32];
  double bb = 0, zr = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n3; i += gridDim.x * blockDim.x) {
    const double bi = b[i];
    const float rv = (float)bi, dv = (float)dinv[i], zv = dv * rv;
    x[i] = 0;
    r32[i] = rv;
    dinv32[i] = dv;
    p32[i] = zv;
    d32[i] = 0.f;
    bb += bi * bi;
    zr += (double)zv * (double)rv;
  }
  const double s1 = block_sum(bb, sh), s2 = block_sum(zr, sh);
  if (threadIdx.x == 0) { partial[2 * blockIdx.x] = s1; partial[2 * blockIdx.x + 1] = s2; }
  if (!last_block(&st->counter)) return;
  double tt[2];
  sum_partials<2>(partial, gridDim.x, tt, sh);
  const double tb = tt[0], tz = tt[1];
  if (threadIdx.x == 0) {
    st->bnorm = sqrt(tb);
    st->zr = tz;
    st->beta = 0; st->alpha = 0; st->err = 0;
    st->it = 0; st->iterations = 0; st->matvecs = 0; st->status = 0;
    st->done = (st->bnorm > 1e-25) ? 0 : 1;  // SolverPCG.cs:112
    st->need = 0; st->err_ref = 1.0;
    st->counter = 0;
  }
}

// x += d, d = 0 (the FP32 correction into the FP64 iterate)
__global__ void k_pcgm_fold(int n3, double* __restrict__ x, float* __restrict__ d32) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n3; i += gridDim.x * blockDim.x) {
    x[i] += (double)d32[i];
    d32[i] = 0.f;
  }
}

// FP64 true residual r = b - y (y = K x with the FP64 values) into the FP32 r:
// stop when ||r||/||b|| < tol, else gamma = (D r).r and the loop resumes with
// its direction.
__global__ void __launch_bounds__(kPcgThreads) k_pcgm_true(int n3, const double* __restrict__ b,
                                                           const double* __restrict__ y,
                                                           const float* __restrict__ dinv32, float* __restrict__ r32,
                                                           double* __restrict__ partial, PcgState* st) {
  __shared__ double sh[32];
  double rr = 0, zr = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n3; i += gridDim.x * blockDim.x) {
    const double ri = b[i] - y[i];
    const float rv = (float)ri;
    r32[i] = rv;
    rr += ri * ri;
    zr += (double)(dinv32[i] * rv) * (double)rv;
  }
  const double s1 = block_sum(rr, sh), s2 = block_sum(zr, sh);
  if (threadIdx.x == 0) { partial[2 * blockIdx.x] = s1; partial[2 * blockIdx.x + 1] = s2; }
  if (!last_block(&st->counter)) return;
  double tt[2];
  sum_partials<2>(partial, gridDim.x, tt, sh);
  const double tr = tt[0], tz = tt[1];
  if (threadIdx.x == 0) {
    const int it = st->it;
    st->err = sqrt(tr) / st->bnorm;
    st->need = 0;
    if (st->err < st->tol) {
      st->done = 1; st->iterations = it;
    } else if (it + 1 >= st->max_it) {
      st->done = 1; st->iterations = st->max_it; st->status = MSG_ERR_NOT_CONVERGED;
    } else {
      st->zr = tz;
      st->it = it + 1;
      st->err_ref = st->err;
      st->done = 0;
    }
    st->counter = 0;
  }
}

__global__ void __launch_bounds__(kPcgThreads) k_pcg_update(int n_rows, const double* __restrict__ dinv,
                                                            double* __restrict__ r, double* __restrict__ x,
                                                            const double* __restrict__ p0,
                                                            const double* __restrict__ p1,
                                                            const double* __restrict__ q, double* __restrict__ partial,
                                                            PcgState* st) {
  __shared__ double sh[32];
  if (st->done) return;
  const int it = st->it;
  const double alpha = st->alpha;
  const double* __restrict__ pnew = (it & 1) ? p0 : p1;
  double rr = 0, zr = 0;
  // two components a thread at a time (double2; the vectors start at 16-byte boundaries)
  const int n3 = 3 * n_rows, n2 = n3 >> 1;
  const int tid = blockIdx.x * blockDim.x + threadIdx.x, nt = gridDim.x * blockDim.x;
  for (int i = tid; i < n2; i += nt) {
    const double2 rv = reinterpret_cast<const double2*>(r)[i], qv = reinterpret_cast<const double2*>(q)[i];
    const double2 xv = reinterpret_cast<const double2*>(x)[i], pv = reinterpret_cast<const double2*>(pnew)[i];
    const double2 dv = reinterpret_cast<const double2*>(dinv)[i];
    const double r0 = rv.x - alpha * qv.x, r1 = rv.y - alpha * qv.y;
    reinterpret_cast<double2*>(r)[i] = make_double2(r0, r1);
    reinterpret_cast<double2*>(x)[i] = make_double2(xv.x + alpha * pv.x, xv.y + alpha * pv.y);
    rr += r0 * r0;
    zr += dv.x * r0 * r0;
    rr += r1 * r1;
    zr += dv.y * r1 * r1;
  }
  for (int i = 2 * n2 + tid; i < n3; i += nt) {
    const double ri = r[i] - alpha * q[i];
    r[i] = ri;
    x[i] = x[i] + alpha * pnew[i];
    rr += ri * ri;
    zr += dinv[i] * ri * ri;
  }
  double s1 = block_sum(rr, sh);
  double s2 = block_sum(zr, sh);
  if (threadIdx.x == 0) { partial[2 * blockIdx.x] = s1; partial[2 * blockIdx.x + 1] = s2; }
  if (!last_block(&st->counter)) return;
  double tt[2];
  sum_partials<2>(partial, gridDim.x, tt, sh);
  const double tr = tt[0], tz = tt[1];
  if (threadIdx.x == 0) {
    st->err = sqrt(tr) / st->bnorm;
    if (st->err < st->tol) {
      st->done = 1; st->iterations = it;
    } else if (it + 1 >= st->max_it) {
      st->done = 1; st->iterations = st->max_it; st->status = MSG_ERR_NOT_CONVERGED;
    } else {
      st->beta = tz / st->zr;
      st->zr = tz;
      st->it = it + 1;
    }
    st->counter = 0;
  }
}

__global__ void k_to_f32(size_t n, const double* __restrict__ a, float* __restrict__ b) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    b[i] = (float)a[i];
}

}  // namespace

int launch_to_f32(Context* ctx, size_t n, const double* a, float* b) {
  k_to_f32<<<ctx->sm_count * 8, 256, 0, ctx->stream>>>(n, a, b);
  count_launch(ctx);
  MSG_CUDA(ctx, cudaGetLastError());
  return MSG_OK;
}

int launch_bsr_assemble(Context* ctx, const Mesh* m, const double* d_Ke, double* d_val) {
  const int64_t n_pos = m->pat.n_slots * 32;
  if (n_pos == 0) return MSG_OK;
  const int64_t nt = n_pos * 9;
  k_bsr_assemble<<<(unsigned)((nt + 255) / 256), 256, 0, ctx->stream>>>(
      n_pos, m->d_col.as<int>(), m->d_contrib_ptr.as<int64_t>(), m->d_contrib.as<int>(), d_Ke, d_val);
  k_bsr_mask<<<(m->n_nodes + 127) / 128, 128, 0, ctx->stream>>>(m->n_nodes, m->d_slice_ptr.as<int64_t>(),
                                                                m->d_col.as<int>(), m->d_mask.as<uint8_t>(), d_val);
  count_launch(ctx, 2);
  MSG_CUDA(ctx, cudaGetLastError());
  return MSG_OK;
}

int launch_bsr_diag_inv(Context* ctx, const Mesh* m, const double* d_val, double* d_dinv) {
  k_bsr_diag_inv<<<(m->n_nodes + 127) / 128, 128, 0, ctx->stream>>>(m->n_nodes, m->d_diag_pos.as<int>(), d_val,
                                                                    d_dinv);
  count_launch(ctx);
  MSG_CUDA(ctx, cudaGetLastError());
  return MSG_OK;
}

int launch_bsr_spmv(Context* ctx, const Mesh* m, const double* d_val, const double* d_x, double* d_y) {
  k_bsr_spmv3<<<m->pat.n_slices, 96, 0, ctx->stream>>>(m->n_nodes, m->d_slice_ptr.as<int64_t>(), m->d_col.as<int>(),
                                                        d_val, d_x, d_y);
  count_launch(ctx);
  MSG_CUDA(ctx, cudaGetLastError());
  return MSG_OK;
}

int launch_dof_to_node(Context* ctx, const Mesh* m, const double* d_in, double* d_out, int n_vec, int64_t in_stride,
                       int64_t out_stride) {
  if (m->n_dofs == 0 || n_vec == 0) return MSG_OK;
  dim3 grid((m->n_dofs + 255) / 256, n_vec);
  k_dof_to_node<<<grid, 256, 0, ctx->stream>>>(m->n_dofs, m->d_free_rows.as<int>(), d_in, d_out, in_stride,
                                               out_stride);
  count_launch(ctx);
  MSG_CUDA(ctx, cudaGetLastError());
  return MSG_OK;
}

int launch_node_to_dof(Context* ctx, const Mesh* m, const double* d_in, double* d_out, int n_vec, int64_t in_stride,
                       int64_t out_stride) {
  if (m->n_dofs == 0 || n_vec == 0) return MSG_OK;
  dim3 grid((m->n_dofs + 255) / 256, n_vec);
  k_node_to_dof<<<grid, 256, 0, ctx->stream>>>(m->n_dofs, m->d_free_rows.as<int>(), d_in, d_out, in_stride,
                                               out_stride);
  count_launch(ctx);
  MSG_CUDA(ctx, cudaGetLastError());
  return MSG_OK;
}

// The FP64 loop's direction + SpMV launch (shape chosen by size).
static void launch_pcg_dir_spmv(Context* ctx, const Mesh* m, double* v64, double* dv, double* rv, double* p0,
                                double* p1, double* qv, double* pa, PcgState* st, cudaStream_t stream) {
  const int nr = m->n_nodes;
  const int ns = m->pat.n_slices;
  const bool small = ns < ctx->sm_count * 32;  // fewer slices than 32 warps per SM: 4 warps per slice
  const int64_t* sp = m->d_slice_ptr.as<int64_t>();
  const int* cl = m->d_col.as<int>();
  // FP64 values stream through with evict-first loads (measured faster at every size)
  if (small)
    k_pcg_dir_spmv_rows<double, 1, 4, true><<<ns, 128, 0, stream>>>(nr, ns, sp, cl, v64, dv, rv, p0, p1, qv, pa, st);
  else
    k_pcg_dir_spmv_rows<double, 8, 1, true><<<(ns + 7) / 8, 256, 0, stream>>>(nr, ns, sp, cl, v64, dv, rv, p0, p1, qv,
                                                                              pa, st);
}

// The mixed loop's FP32 SpMV launch: small matrices one slice per CTA with 4
// warps; large ones by the "spmv32_shape" option (slots per group / slices per
// CTA: 0: 4 / 8, 1: 8 / 8, 2: 4 / 4, 3: 8 / 4). FP32 values of matrices up to
// ~60 % of L2 stay there across iterations, larger ones stream (evict-first).
static void launch_pcgm_spmv(Context* ctx, const Mesh* m, const float* v32, const float* p32, const float* r32,
                             const float* dinv32, float* q32, double* pa, PcgState* st, cudaStream_t stream) {
  const int nr = m->n_nodes;
  const int ns = m->pat.n_slices;
  const bool small = ns < ctx->sm_count * 32;
  const int64_t* sp = m->d_slice_ptr.as<int64_t>();
  const int* cl = m->d_col.as<int>();
  const bool strm = (size_t)m->pat.n_slots * 32 * 9 * 4 > (size_t)76 << 20;
  const int shape = ctx->spmv32_shape;
  // persistent grid (W = 1): the resident CTAs of every SM once
  auto fill = [&](const void* k, int threads, int n_ctas) {
    int occ = 1;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k, threads, 0) != cudaSuccess || occ < 1) occ = 1;
    return std::max(1, std::min(n_ctas, ctx->sm_count * occ));
  };
#define MSG_SPMV32(S, W, U)                                                                                       \
  do {                                                                                                           \
    const int grid = W > 1 ? (ns + S - 1) / S                                                                    \
                           : fill((const void*)k_pcgm_spmv<S, W, true, U>, 32 * S * W, (ns + S - 1) / S);        \
    if (strm)                                                                                                    \
      k_pcgm_spmv<S, W, true, U><<<grid, 32 * S * W, 0, stream>>>(nr, ns, sp, cl, v32, p32, r32, dinv32, q32, pa, \
                                                                  st);                                           \
    else                                                                                                         \
      k_pcgm_spmv<S, W, false, U><<<grid, 32 * S * W, 0, stream>>>(nr, ns, sp, cl, v32, p32, r32, dinv32, q32,    \
                                                                   pa, st);                                      \
  } while (0)
  if (small) MSG_SPMV32(1, 4, 4);
  else if (shape == 1) MSG_SPMV32(8, 1, 8);
  else if (shape == 2) MSG_SPMV32(4, 1, 4);
  else if (shape == 3) MSG_SPMV32(4, 1, 8);
  else MSG_SPMV32(8, 1, 4);
#undef MSG_SPMV32
}

// The device loop's control (one thread each, inside the solve's graph):
// another round of iterations while the solve runs, at most
// max_it / chunk + 2 max_it + 4 rounds (every round but a paused one advances
// the iteration count, every pause ends or advances it, so the bound is never
// the reason to stop); and, in the mixed loop, the FP64 true-residual step
// when the round paused for one.
__global__ void k_pcg_loop_while(PcgState* st, cudaGraphConditionalHandle h, int chunk) {
  const long long r = ++st->rounds;
  const long long cap = (long long)st->max_it / chunk + 2LL * st->max_it + 4;
  cudaGraphSetConditional(h, (!st->done && r < cap) ? 1u : 0u);
}

__global__ void k_pcg_loop_if(PcgState* st, cudaGraphConditionalHandle h) {
  const int need = st->need;
  if (need) st->pauses += 1;
  cudaGraphSetConditional(h, need ? 1u : 0u);
}

// Runs the device PCG on node-layout vectors, the whole solve one graph
// launch: a WHILE node repeats a round of `chunk` iterations (2 kernels each,
// captured once per matrix) until the state says done, with no host round
// trip between rounds. Kernels after convergence return immediately, so the
// recorded iteration count is exact. Mixed precision: the FP32 loop
// (k_pcgm_*); when it pauses (need), an IF node runs x += d, y = K x with the
// FP64 values and k_pcgm_true, which replace the recursive residual (or end
// the solve on the true residual).
int pcg_solve_device(Context* ctx, Matrix* A, const double* d_b, double* d_x, int max_it, double tol, int* iterations,
                     double* rel_res, int* status, bool mixed) {
  Mesh* m = A->mesh;
  const int nr = m->n_nodes;
  const int n = 3 * nr;
  cudaStream_t s = ctx->stream;
  MSG_TRY(context_resources(ctx));
  if (!A->d_r.ptr) {
    MSG_TRY(A->d_r.alloc(ctx, sizeof(double) * n));
    MSG_TRY(A->d_p0.alloc(ctx, sizeof(double) * n));
    MSG_TRY(A->d_p1.alloc(ctx, sizeof(double) * n));
    MSG_TRY(A->d_q.alloc(ctx, sizeof(double) * n));
    // partials: one per FP64 SpMV CTA (slice), three per FP32 SpMV CTA or two per update CTA
    MSG_TRY(A->d_partial.alloc(ctx, sizeof(double) * std::max<size_t>(2 * 4096, 3 * (size_t)m->pat.n_slices)));
    MSG_TRY(A->d_state.alloc(ctx, sizeof(PcgState)));
    MSG_CUDA(ctx, cudaMemsetAsync(A->d_state.ptr, 0, sizeof(PcgState), s));
  }
  if (mixed && !A->d_val32.ptr) {
    const size_t nv = (size_t)m->pat.n_slots * 32 * 9;
    MSG_TRY(A->d_val32.alloc(ctx, sizeof(float) * std::max<size_t>(1, nv)));
    MSG_TRY(A->d_tmp.alloc(ctx, sizeof(double) * n));   // y = K x of the true residual
    MSG_TRY(A->d_tmp2.alloc(ctx, sizeof(float) * n));   // p (FP32)
    MSG_TRY(A->d_m32.alloc(ctx, sizeof(float) * 4 * (((size_t)n + 31) / 32 * 32)));
    k_to_f32<<<ctx->sm_count * 8, 256, 0, s>>>(nv, A->d_val.as<double>(), A->d_val32.as<float>());
    count_launch(ctx);
  }
  PcgState* st = A->d_state.as<PcgState>();
  const int grid_v = std::min(4096, std::max(1, std::min((n + kPcgThreads - 1) / kPcgThreads, ctx->sm_count * 8)));
  // the update passes: float4 (mixed) or double2 (FP64) a thread, at most 4 CTAs an SM
  const int grid_u = std::max(1, std::min((n / (mixed ? 4 : 2) + kPcgThreads - 1) / kPcgThreads, ctx->sm_count * 4));
  double* pa = A->d_partial.as<double>();
  float *p32 = nullptr, *r32 = nullptr, *q32 = nullptr, *d32 = nullptr, *dinv32 = nullptr;
  if (mixed) {
    const size_t n32 = ((size_t)n + 31) / 32 * 32;  // 128-byte aligned vectors
    p32 = A->d_tmp2.as<float>();
    r32 = A->d_m32.as<float>();
    q32 = r32 + n32;
    d32 = q32 + n32;
    dinv32 = d32 + n32;
    k_pcgm_init<<<grid_v, kPcgThreads, 0, s>>>(n, d_b, A->d_dinv.as<double>(), d_x, r32, p32, d32, dinv32, pa, st);
  } else {
    k_pcg_init<<<grid_v, kPcgThreads, 0, s>>>(nr, d_b, A->d_dinv.as<double>(), A->d_r.as<double>(), d_x,
                                              A->d_p0.as<double>(), A->d_p1.as<double>(), pa, st);
  }
  count_launch(ctx);
  // tol, max_it and the mixed-precision settings into the state (after init so the counter reset does not race)
  {
    const int mx = mixed ? 1 : 0;
    const double delta = ctx->reliable_delta;
    MSG_CUDA(ctx, cudaMemcpyAsync(&st->tol, &tol, sizeof(double), cudaMemcpyHostToDevice, s));
    MSG_CUDA(ctx, cudaMemcpyAsync(&st->max_it, &max_it, sizeof(int), cudaMemcpyHostToDevice, s));
    MSG_CUDA(ctx, cudaMemcpyAsync(&st->mixed, &mx, sizeof(int), cudaMemcpyHostToDevice, s));
    MSG_CUDA(ctx, cudaMemcpyAsync(&st->delta, &delta, sizeof(double), cudaMemcpyHostToDevice, s));
    // the pageable copies above are staged before they return
  }
  const int chunk = 8;
  const int graph_kind = mixed ? 1 + ctx->spmv32_shape : 0;  // the captured loop's kernels and shapes
  if (!A->graph || A->graph_chunk != chunk || A->graph_x != (const void*)d_x || A->graph_mixed != graph_kind ||
      (mixed && A->graph_b != (const void*)d_b)) {
    if (A->graph) { cudaGraphExecDestroy(A->graph); A->graph = nullptr; }
    struct Graphs {
      cudaGraph_t round = nullptr, pause = nullptr, loop = nullptr;
      ~Graphs() {
        if (round) cudaGraphDestroy(round);
        if (pause) cudaGraphDestroy(pause);
        if (loop) cudaGraphDestroy(loop);
      }
    } G;
    // one round: `chunk` iterations
    MSG_CUDA(ctx, cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    for (int k = 0; k < chunk; ++k) {
      if (mixed) {
        launch_pcgm_spmv(ctx, m, A->d_val32.as<float>(), p32, r32, dinv32, q32, pa, st, s);
        k_pcgm_update<<<grid_u, kPcgThreads, 0, s>>>(n, dinv32, r32, p32, q32, d32, pa, st);
      } else {
        launch_pcg_dir_spmv(ctx, m, A->d_val.as<double>(), A->d_dinv.as<double>(), A->d_r.as<double>(),
                            A->d_p0.as<double>(), A->d_p1.as<double>(), A->d_q.as<double>(), pa, st, s);
        k_pcg_update<<<grid_u, kPcgThreads, 0, s>>>(nr, A->d_dinv.as<double>(), A->d_r.as<double>(), d_x,
                                                    A->d_p0.as<double>(), A->d_p1.as<double>(), A->d_q.as<double>(),
                                                    pa, st);
      }
    }
    MSG_CUDA(ctx, cudaStreamEndCapture(s, &G.round));
    if (mixed) {
      // the pause: x += d in FP64, y = K x, the true residual (resume or stop)
      MSG_CUDA(ctx, cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
      k_pcgm_fold<<<grid_v, kPcgThreads, 0, s>>>(n, d_x, d32);
      k_bsr_spmv3<<<m->pat.n_slices, 96, 0, s>>>(nr, m->d_slice_ptr.as<int64_t>(), m->d_col.as<int>(),
                                                  A->d_val.as<double>(), d_x, A->d_tmp.as<double>());
      k_pcgm_true<<<grid_v, kPcgThreads, 0, s>>>(n, d_b, A->d_tmp.as<double>(), dinv32, r32, pa, st);
      MSG_CUDA(ctx, cudaStreamEndCapture(s, &G.pause));
    }
    MSG_CUDA(ctx, cudaGraphCreate(&G.loop, 0));
    cudaGraphConditionalHandle h_while = 0, h_if = 0;
    MSG_CUDA(ctx, cudaGraphConditionalHandleCreate(&h_while, G.loop, 1, cudaGraphCondAssignDefault));
    cudaGraphNodeParams wp = {};
    wp.type = cudaGraphNodeTypeConditional;
    wp.conditional.handle = h_while;
    wp.conditional.type = cudaGraphCondTypeWhile;
    wp.conditional.size = 1;
    cudaGraphNode_t wn = nullptr, last = nullptr;
    MSG_CUDA(ctx, cudaGraphAddNode(&wn, G.loop, nullptr, 0, &wp));
    cudaGraph_t body = wp.conditional.phGraph_out[0];
    MSG_CUDA(ctx, cudaGraphAddChildGraphNode(&last, body, nullptr, 0, G.round));
    auto add_kernel = [&](void* fn, void** args) -> int {
      cudaKernelNodeParams kp = {};
      kp.func = fn;
      kp.gridDim = dim3(1);
      kp.blockDim = dim3(1);
      kp.kernelParams = args;
      cudaGraphNode_t kn = nullptr;
      MSG_CUDA(ctx, cudaGraphAddKernelNode(&kn, body, &last, 1, &kp));
      last = kn;
      return MSG_OK;
    };
    if (mixed) {
      MSG_CUDA(ctx, cudaGraphConditionalHandleCreate(&h_if, body, 0, 0));
      void* a_if[] = {&st, &h_if};
      MSG_TRY(add_kernel((void*)k_pcg_loop_if, a_if));
      cudaGraphNodeParams ip = {};
      ip.type = cudaGraphNodeTypeConditional;
      ip.conditional.handle = h_if;
      ip.conditional.type = cudaGraphCondTypeIf;
      ip.conditional.size = 1;
      cudaGraphNode_t in = nullptr, pn = nullptr;
      MSG_CUDA(ctx, cudaGraphAddNode(&in, body, &last, 1, &ip));
      MSG_CUDA(ctx, cudaGraphAddChildGraphNode(&pn, ip.conditional.phGraph_out[0], nullptr, 0, G.pause));
      last = in;
    }
    int chunk_arg = chunk;
    void* a_while[] = {&st, &h_while, &chunk_arg};
    MSG_TRY(add_kernel((void*)k_pcg_loop_while, a_while));
    cudaError_t e = cudaGraphInstantiate(&A->graph, G.loop, 0);
    if (e != cudaSuccess) {
      A->graph = nullptr;
      return cuda_error(ctx, e, "cudaGraphInstantiate");
    }
    A->graph_chunk = chunk;
    A->graph_x = d_x;
    A->graph_b = d_b;
    A->graph_mixed = graph_kind;
  }
  MSG_CUDA(ctx, cudaMemsetAsync(&st->rounds, 0, 2 * sizeof(int), s));  // rounds, pauses
  {
    cudaError_t e = cudaGraphLaunch(A->graph, s);
    if (e != cudaSuccess) return cuda_error(ctx, e, "cudaGraphLaunch");
  }
  if (mixed) {  // a correction left by a solve that ended without a true residual
    k_pcgm_fold<<<grid_v, kPcgThreads, 0, s>>>(n, d_x, d32);
    count_launch(ctx);
  }
  MSG_CUDA(ctx, cudaGetLastError());
  PcgState hs;
  MSG_CUDA(ctx, cudaMemcpyAsync(&hs, st, sizeof(PcgState), cudaMemcpyDeviceToHost, s));
  MSG_CUDA(ctx, cudaStreamSynchronize(s));
  count_launch(ctx, hs.rounds * (2 * chunk + (mixed ? 2 : 1)) + 3 * hs.pauses);
  if (iterations) *iterations = hs.iterations;
  if (rel_res) *rel_res = hs.err;
  if (status) *status = hs.done ? hs.status : MSG_ERR_NOT_CONVERGED;
  return MSG_OK;
}

// ------------------------------------------------------------------ PCG without allocation
// Scratch of MSG_PCG_SOLVE_NOALLOC: a fixed array in device memory, so the call
// needs no cudaMalloc. Sized for meshes of up to kNoAllocMaxNodes nodes: six
// node-layout FP64 vectors (b, x, r, two search directions, K p), the per-CTA
// partial sums and the scalar state, about 9.5 MB. Every GPU that loads the
// library holds this array until the process exits.
constexpr int kNoAllocMaxNodes = 65536;
constexpr size_t kNoAllocVecBytes = sizeof(double) * 3 * (size_t)kNoAllocMaxNodes;
constexpr size_t kNoAllocPartials = 2 * 4096;  // >= max(2 * update CTAs, slices of 65536 nodes)
constexpr size_t kNoAllocStateOff = 6 * kNoAllocVecBytes + sizeof(double) * kNoAllocPartials;
constexpr size_t kNoAllocBytes = kNoAllocStateOff + 256;
static_assert(sizeof(PcgState) <= 256, "the scalar state fits its slot of the scratch");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

// Device address of the scratch array on the current device (host code cannot
// use the array's name as a device address). MSG_CREATE looks it up once per
// context, with the context's device current, so no solve call triggers the
// module load that the first lookup may cause.
cudaError_t noalloc_scratch_address(unsigned char** out) {
  void* p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  *out = static_cast<unsigned char*>(p);
  return e;
}

}  // namespace msg

using namespace msg;

// The device Jacobi-PCG of MSG_PCG_SOLVE, for callers that must not allocate
// device memory during the solve: the solve's working vectors live in the
// fixed scratch array above instead of buffers from cudaMalloc, and the
// right-hand side and solution are the caller's device buffers. Kernels and
// their order are those of MSG_PCG_SOLVE, launched one by one.
extern "C" int MSG_PCG_SOLVE_NOALLOC(MSG_MAT A, const double* b_dev, double* x_dev, int max_it, double tol,
                                     int* iterations, double* rel_res) {
  if (!A || !b_dev || !x_dev || max_it <= 0 || !(tol > 0)) return MSG_ERR_INVALID_ARGUMENT;
  Mesh* m = A->mesh;
  Context* ctx = m->ctx;
  std::lock_guard<std::recursive_mutex> lk(ctx->mu);
  MSG_CUDA(ctx, cudaSetDevice(ctx->device));
  const int nr = m->n_nodes;
  if (nr > kNoAllocMaxNodes)
    return set_error(ctx, MSG_ERR_INVALID_ARGUMENT,
                     "MSG_PCG_SOLVE_NOALLOC: mesh has %d nodes, the fixed scratch holds at most %d", nr,
                     kNoAllocMaxNodes);
  unsigned char* base = ctx->noalloc_scratch;
  if (!base) return set_error(ctx, MSG_ERR_CUDA, "MSG_PCG_SOLVE_NOALLOC: scratch address not resolved");
  const size_t n = 3 * (size_t)nr;
  double* bn = reinterpret_cast<double*>(base);
  double* xn = reinterpret_cast<double*>(base + kNoAllocVecBytes);
  double* r = reinterpret_cast<double*>(base + 2 * kNoAllocVecBytes);
  double* p0 = reinterpret_cast<double*>(base + 3 * kNoAllocVecBytes);
  double* p1 = reinterpret_cast<double*>(base + 4 * kNoAllocVecBytes);
  double* q = reinterpret_cast<double*>(base + 5 * kNoAllocVecBytes);
  double* partial = reinterpret_cast<double*>(base + 6 * kNoAllocVecBytes);
  PcgState* st = reinterpret_cast<PcgState*>(base + kNoAllocStateOff);
  cudaStream_t s = ctx->stream;
  // the array keeps the previous call's contents: clear what must start at zero
  MSG_CUDA(ctx, cudaMemsetAsync(bn, 0, sizeof(double) * n, s));
  MSG_CUDA(ctx, cudaMemsetAsync(st, 0, sizeof(PcgState), s));
  MSG_TRY(launch_dof_to_node(ctx, m, b_dev, bn, 1, 0, 0));
  const int grid_v = std::min(4096, std::max(1, std::min((int)((n + kPcgThreads - 1) / kPcgThreads), ctx->sm_count * 8)));
  k_pcg_init<<<grid_v, kPcgThreads, 0, s>>>(nr, bn, A->d_dinv.as<double>(), r, xn, p0, p1, partial, st);
  count_launch(ctx);
  MSG_CUDA(ctx, cudaMemcpyAsync(&st->tol, &tol, sizeof(double), cudaMemcpyHostToDevice, s));
  MSG_CUDA(ctx, cudaMemcpyAsync(&st->max_it, &max_it, sizeof(int), cudaMemcpyHostToDevice, s));
  int done = 0;
  for (int it = 0; it < max_it + 8 && !done; it += 8) {
    for (int k = 0; k < 8; ++k) {
      launch_pcg_dir_spmv(ctx, m, A->d_val.as<double>(), A->d_dinv.as<double>(), r, p0, p1, q, partial, st, s);
      k_pcg_update<<<grid_v, kPcgThreads, 0, s>>>(nr, A->d_dinv.as<double>(), r, xn, p0, p1, q, partial, st);
    }
    count_launch(ctx, 16);
    MSG_CUDA(ctx, cudaMemcpyAsync(&done, &st->done, sizeof(int), cudaMemcpyDeviceToHost, s));
    MSG_CUDA(ctx, cudaStreamSynchronize(s));
  }
  MSG_CUDA(ctx, cudaGetLastError());
  MSG_TRY(launch_node_to_dof(ctx, m, xn, x_dev, 1, 0, 0));
  PcgState hs;
  MSG_CUDA(ctx, cudaMemcpyAsync(&hs, st, sizeof(PcgState), cudaMemcpyDeviceToHost, s));
  MSG_CUDA(ctx, cudaStreamSynchronize(s));
  if (iterations) *iterations = hs.iterations;
  if (rel_res) *rel_res = hs.err;
  if (hs.status != MSG_OK)
    return set_error(ctx, hs.status,
                     hs.status == MSG_ERR_BREAKDOWN ? "PCG breakdown (p.q <= 0 or NaN)" : "PCG did not converge");
  return MSG_OK;
}
