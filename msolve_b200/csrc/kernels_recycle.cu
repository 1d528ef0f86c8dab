// PCG with re-orthogonalised search vectors kept across solves, the device
// twin of SolverPCG (ISAAR.MSolve.Solvers/PCG/SolverPCG.cs:105-149) driven by
// SolverPCGReorthogonalizationSearchVectorCalculator
// (ISAAR.MSolve.Solvers/PCG/SolverPCGReorthogonalizationSearchVectorCalculator.cs:11-65)
// over SearchVectors (ISAAR.MSolve.Solvers/SearchVectors.cs:13-166):
//   p = z - sum_c (z.q_c / p_c.q_c) p_c over every stored pair (classical
//       Gram-Schmidt against the directions of this and earlier solves),
//   q = K p, alpha = (p.r)/(p.q), the pair (p, q) is appended to the store,
//   r -= alpha q, x += alpha p, stop on ||r||/||b||.
// The starting vector from the store (InitializeStartingVectorFromSearchVectors:
// the last pair is dropped, then x0 = sum_c (p_c.b / p_c.q_c) p_c) is followed by
// r0 = b - K x0 (the reference defines the starting vector but never wires it
// into a solve); with start mode 2 the store is emptied after x0, so a matrix
// other than the one that produced the pairs starts a fresh Krylov space.
// The store lives on the device: P and Q [capacity][3 n_nodes] (node layout,
// constrained components 0) and p_c.q_c; every reduction runs in a fixed
// order, so results do not depend on timing. Jacobi preconditioner, the
// matrix's FP64 values.
#include "msg_internal.h"

namespace msg {
namespace {

constexpr int kDotThreads = 256;

// out[c] = sum_i V[c][i] * w[i] for c < k (one CTA per vector; strided
// per-thread sums, then a fixed tree).
__global__ void __launch_bounds__(kDotThreads) k_svs_dots(int64_t n, int k, const double* __restrict__ V,
                                                          int64_t ld, const double* __restrict__ w,
                                                          double* __restrict__ out) {
  __shared__ double sh[kDotThreads];
  const int c = blockIdx.x;
  if (c >= k) return;
  const double* v = V + (size_t)c * ld;
  double s = 0.0;
  for (int64_t i = threadIdx.x; i < n; i += kDotThreads) s = fma(v[i], w[i], s);
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int h = kDotThreads / 2; h > 0; h >>= 1) {
    if (threadIdx.x < h) sh[threadIdx.x] += sh[threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[c] = sh[0];
}

// p = z - sum_c (a[c] / pq[c]) P[c] (CalculateReorthogonalizedSearchVector, c in order)
__global__ void k_svs_combine(int64_t n, int k, const double* __restrict__ z, const double* __restrict__ P,
                              int64_t ld, const double* __restrict__ a, const double* __restrict__ pq,
                              double* __restrict__ p) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double v = z[i];
    for (int c = 0; c < k; ++c) v -= (a[c] / pq[c]) * P[(size_t)c * ld + i];
    p[i] = v;
  }
}

// x0 = sum_c (pb[c] / pq[c]) P[c]
__global__ void k_svs_start(int64_t n, int k, const double* __restrict__ P, int64_t ld,
                            const double* __restrict__ pb, const double* __restrict__ pq, double* __restrict__ x) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double v = 0.0;
    for (int c = 0; c < k; ++c) v += (pb[c] / pq[c]) * P[(size_t)c * ld + i];
    x[i] = v;
  }
}

// z = dinv * r
__global__ void k_jacobi(int64_t n, const double* __restrict__ dinv, const double* __restrict__ r,
                         double* __restrict__ z) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    z[i] = dinv[i] * r[i];
}

// r -= alpha q, x += alpha p (alpha on the device); also stores (p, q) into the store slot
__global__ void k_svs_step(int64_t n, const double* __restrict__ alpha, const double* __restrict__ p,
                           const double* __restrict__ q, double* __restrict__ r, double* __restrict__ x,
                           double* __restrict__ Pc, double* __restrict__ Qc) {
  const double a = *alpha;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double pv = p[i], qv = q[i];
    r[i] -= a * qv;
    x[i] += a * pv;
    Pc[i] = pv;
    Qc[i] = qv;
  }
}

// r = b - y
__global__ void k_sub(int64_t n, const double* __restrict__ b, const double* __restrict__ y, double* __restrict__ r) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    r[i] = b[i] - y[i];
}

// alpha = pr / pq; scal = [pr, pq, rr, alpha]
__global__ void k_alpha_scalar(double* scal) {
  if (threadIdx.x == 0 && blockIdx.x == 0) scal[3] = scal[0] / scal[1];
}

}  // namespace

int svs_create(Context* ctx, Mesh* m, int capacity, SearchVectorStore** out) {
  if (capacity <= 0) return set_error(ctx, MSG_ERR_INVALID_ARGUMENT, "search vector store: capacity must be > 0");
  std::unique_ptr<SearchVectorStore> s(new SearchVectorStore());
  s->mesh = m;
  s->n3 = 3 * (int64_t)m->n_nodes;
  s->capacity = capacity;
  MSG_TRY(s->P.alloc(ctx, sizeof(double) * (size_t)capacity * s->n3));
  MSG_TRY(s->Q.alloc(ctx, sizeof(double) * (size_t)capacity * s->n3));
  MSG_TRY(s->pq.alloc(ctx, sizeof(double) * (size_t)capacity));
  MSG_TRY(s->coef.alloc(ctx, sizeof(double) * (size_t)capacity));
  MSG_TRY(s->work.alloc(ctx, sizeof(double) * 6 * (size_t)s->n3));
  MSG_TRY(s->scal.alloc(ctx, sizeof(double) * 8));
  retain(m);
  *out = s.release();
  return MSG_OK;
}

int pcg_reorth_solve(Context* ctx, Matrix* A, SearchVectorStore* S, const double* d_b, double* d_x, int start_mode,
                     int max_it, double tol, int* iterations, double* rel_res) {
  const bool start = start_mode != 0;
  Mesh* m = A->mesh;
  cudaStream_t st = ctx->stream;
  const int64_t n = S->n3, ld = S->n3;
  double* w = S->work.as<double>();
  double *r = w, *z = w + n, *p = w + 2 * n, *q = w + 3 * n, *y = w + 4 * n;
  double* scal = S->scal.as<double>();
  double* P = S->P.as<double>();
  double* Q = S->Q.as<double>();
  double* pq = S->pq.as<double>();
  double* coef = S->coef.as<double>();
  const double* dinv = A->d_dinv.as<double>();
  const int grid = std::min<int64_t>((n + 255) / 256, (int64_t)ctx->sm_count * 8);
  double h[4];
  auto dot = [&](const double* a, const double* b, double* out) {
    k_svs_dots<<<1, kDotThreads, 0, st>>>(n, 1, a, n, b, out);
    count_launch(ctx);
  };
  // ||b|| (InitializeAndGetResidual)
  dot(d_b, d_b, scal + 2);
  MSG_CUDA(ctx, cudaMemcpyAsync(h, scal + 2, sizeof(double), cudaMemcpyDeviceToHost, st));
  MSG_CUDA(ctx, cudaStreamSynchronize(st));
  const double detf = std::sqrt(h[0]);
  if (start && S->count > 0) {
    // InitializeStartingVectorFromReorthogonalizedSearchVectors: drop the last pair
    S->count -= 1;
  }
  if (start && S->count > 0) {
    k_svs_dots<<<S->count, kDotThreads, 0, st>>>(n, S->count, P, ld, d_b, coef);
    k_svs_start<<<grid, 256, 0, st>>>(n, S->count, P, ld, coef, pq, d_x);
    MSG_TRY(launch_bsr_spmv(ctx, m, A->d_val.as<double>(), d_x, y));
    k_sub<<<grid, 256, 0, st>>>(n, d_b, y, r);
    count_launch(ctx, 3);
    if (start_mode == 2) S->count = 0;  // the pairs belong to another matrix: start a fresh store
  } else {
    MSG_CUDA(ctx, cudaMemsetAsync(d_x, 0, sizeof(double) * n, st));
    MSG_CUDA(ctx, cudaMemcpyAsync(r, d_b, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
  }
  dot(r, r, scal + 2);
  MSG_CUDA(ctx, cudaMemcpyAsync(h, scal + 2, sizeof(double), cudaMemcpyDeviceToHost, st));
  MSG_CUDA(ctx, cudaStreamSynchronize(st));
  int its = 0;
  double err = detf > 0 ? std::sqrt(h[0]) / detf : 0.0;
  int status = MSG_OK;
  if (std::sqrt(h[0]) > 1e-25) {
    k_jacobi<<<grid, 256, 0, st>>>(n, dinv, r, z);
    count_launch(ctx);
    int it = 0;
    status = MSG_ERR_NOT_CONVERGED;
    for (; it < max_it; ++it) {
      if (S->count >= S->capacity) {
        status = set_error(ctx, MSG_ERR_OUT_OF_MEMORY, "search vector store is full (%d pairs)", S->capacity);
        break;
      }
      // CalculateReorthogonalizedSearchVector
      if (S->count > 0) {
        k_svs_dots<<<S->count, kDotThreads, 0, st>>>(n, S->count, Q, ld, z, coef);
        k_svs_combine<<<grid, 256, 0, st>>>(n, S->count, z, P, ld, coef, pq, p);
        count_launch(ctx, 2);
      } else {
        MSG_CUDA(ctx, cudaMemcpyAsync(p, z, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
      }
      MSG_TRY(launch_bsr_spmv(ctx, m, A->d_val.as<double>(), p, q));
      // CalculateReorthogonalizedGradient: the pair is stored, alpha = (p.r)/(p.q)
      dot(p, r, scal + 0);
      dot(p, q, scal + 1);
      MSG_CUDA(ctx, cudaMemcpyAsync(pq + S->count, scal + 1, sizeof(double), cudaMemcpyDeviceToDevice, st));
      k_alpha_scalar<<<1, 32, 0, st>>>(scal);
      k_svs_step<<<grid, 256, 0, st>>>(n, scal + 3, p, q, r, d_x, P + (size_t)S->count * ld, Q + (size_t)S->count * ld);
      dot(r, r, scal + 2);
      count_launch(ctx, 2);
      MSG_CUDA(ctx, cudaMemcpyAsync(h, scal, sizeof(double) * 4, cudaMemcpyDeviceToHost, st));
      MSG_CUDA(ctx, cudaStreamSynchronize(st));
      S->count += 1;
      if (!(h[1] == h[1]) || !(h[3] == h[3])) {
        status = set_error(ctx, MSG_ERR_BREAKDOWN, "reorthogonalized PCG breakdown (NaN gradient)");
        break;
      }
      err = std::sqrt(h[2]) / detf;
      if (err < tol) {
        status = MSG_OK;
        break;
      }
      k_jacobi<<<grid, 256, 0, st>>>(n, dinv, r, z);
      count_launch(ctx);
    }
    its = it;
  }
  MSG_CUDA(ctx, cudaGetLastError());
  if (iterations) *iterations = its;
  if (rel_res) *rel_res = err;
  if (status == MSG_ERR_NOT_CONVERGED) return set_error(ctx, status, "reorthogonalized PCG did not converge");
  return status;
}

}  // namespace msg
