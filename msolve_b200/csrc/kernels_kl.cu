// Lognormal Young's-modulus field from a separable Karhunen-Loeve table, the
// device twin of LognormalFileStochasticCoefficientsProvider.GetCoefficient
// (ISAAR.MSolve.PreProcessor/Stochastic/LognormalFileStochasticCoefficientsProvider.cs:134-193)
// evaluated at element bounding-box centres (Hexa8WithStochasticMaterial.cs:112-140),
// or the Gaussian field of GaussianFileStochasticCoefficientsProvider.GetCoefficient
// (GaussianFileStochasticCoefficientsProvider.cs:72-108): E = mean (1 + sum_k xi_k psi_k)
// with the same psi (its sigma is the provider's covariance).
//
// psi[k][e] = sigma sqrt(eig_k) prod_a amp_ka {cos|sin}(w_ka (x_ea - L_a/2)) is
// built once per mesh and table (FP64). The field for R realizations is then
// the product [R x K] . [K x n_e] followed by exp:
//   E[e][r] = exp(mu + sum_k xi[r][k] psi[k][e]).
// A CTA stages a 32-realization x 32-element tile of xi and psi in shared
// memory; each thread produces four (element, realization) values, written
// realization-innermost (coalesced) in FP64 and FP32, and optionally in the
// per-realization layout [r][e] used by the assembled FP64 path.
#include <cstring>

#include "msg_internal.h"

namespace msg {
namespace {

constexpr int kMaxTerms = 64;  // 2 x 64 x 33 doubles of shared memory

__global__ void k_kl_psi(int ne, int K, const double* __restrict__ cen, const double* __restrict__ tab,
                         double L0, double L1, double L2, double sigma, double* __restrict__ psi) {
  // tab rows: [w0 w1 w2 a0 a1 a2 idx0 idx1 idx2 eig] per term
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  const int k = blockIdx.y;
  if (e >= ne) return;
  const double* t = tab + 10 * k;
  double f = sigma * sqrt(t[9]);
  const double L[3] = {L0, L1, L2};
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const double x = cen[3 * e + a] - L[a] / 2;
    const int idx = (int)t[6 + a];
    f *= (idx % 2 == 0) ? t[3 + a] * sin(t[a] * x) : t[3 + a] * cos(t[a] * x);
  }
  psi[(size_t)k * ne + e] = f;
}

__global__ void __launch_bounds__(256) k_kl_field(int ne, int K, int R, int Rp, const double* __restrict__ xi,
                                                  const double* __restrict__ psi, double mu, int gaussian, double mean,
                                                  double* __restrict__ E64_er, float* __restrict__ E32_er,
                                                  double* __restrict__ E64_re, const int* __restrict__ elem_row) {
  __shared__ double s_xi[kMaxTerms][33];
  __shared__ double s_psi[kMaxTerms][33];
  const int tx = threadIdx.x, ty = threadIdx.y;  // 32 x 8
  const int e0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
  for (int k = ty; k < K; k += 8) {
    const int r = r0 + tx;
    s_xi[k][tx] = (r < R) ? xi[(size_t)r * K + k] : 0.0;
    const int e = e0 + tx;
    s_psi[k][tx] = (e < ne) ? psi[(size_t)k * ne + e] : 0.0;
  }
  __syncthreads();
  const int r = r0 + tx;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int le = ty + 8 * q, e = e0 + le;
    if (e >= ne) continue;
    double s = gaussian ? 0.0 : mu;
    for (int k = 0; k < K; ++k) s += s_xi[k][tx] * s_psi[k][le];
    const double E = (r < R) ? (gaussian ? mean * (1.0 + s) : exp(s)) : 1.0;
    const size_t row = elem_row ? (size_t)elem_row[e] : (size_t)e;
    if (E64_er) E64_er[row * Rp + r] = E;
    if (E32_er) E32_er[row * Rp + r] = (float)E;
    if (E64_re && r < R) E64_re[(size_t)r * ne + e] = E;
  }
}

// E of a list of realization slots (one thread per element and slot):
// E[row(e)*Rp + slot] = exp(mu + sum_k xi[i][k] psi[k][e]) in FP64 and FP32,
// the same expression as k_kl_field. xi [n_slots][K].
__global__ void k_kl_field_slots(int ne, int K, int n_slots, const int* __restrict__ slots,
                                 const double* __restrict__ xi, const double* __restrict__ psi, double mu,
                                 int gaussian, double mean, int Rp, double* __restrict__ E64, float* __restrict__ E32,
                                 const int* __restrict__ elem_row) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = blockIdx.y;
  if (e >= ne || i >= n_slots) return;
  const double* x = xi + (size_t)i * K;
  double s = gaussian ? 0.0 : mu;
  for (int k = 0; k < K; ++k) s += x[k] * psi[(size_t)k * ne + e];
  const double E = gaussian ? mean * (1.0 + s) : exp(s);
  const size_t o = (size_t)elem_row[e] * Rp + slots[i];
  E64[o] = E;
  E32[o] = (float)E;
}

}  // namespace

int launch_kl_field_slots(cudaStream_t st, const Mesh* m, const KLDevice* kl, int n_slots, const int* d_slots,
                          const double* d_xi, int Rp, double* d_E64, float* d_E32) {
  dim3 grid((m->n_elems + 127) / 128, n_slots);
  k_kl_field_slots<<<grid, 128, 0, st>>>(m->n_elems, kl->n_terms, n_slots, d_slots, d_xi, kl->psi, kl->mu,
                                         kl->gaussian, kl->mean, Rp, d_E64, d_E32, m->d_pad_elem_row.as<int>());
  return cudaGetLastError() == cudaSuccess ? MSG_OK : MSG_ERR_CUDA;
}

int kl_prepare(Context* ctx, const Mesh* m, const MSG_KL* kl, KLDevice* out) {
  const int K = kl->n_terms;
  if (K <= 0 || K > kMaxTerms) return set_error(ctx, MSG_ERR_INVALID_ARGUMENT, "n_terms must be in 1..%d", kMaxTerms);
  if (!(kl->mean > 0)) return set_error(ctx, MSG_ERR_INVALID_ARGUMENT, "KL mean must be > 0");
  std::vector<double> tab(10 * (size_t)K);
  for (int k = 0; k < K; ++k) {
    for (int a = 0; a < 3; ++a) {
      tab[10 * k + a] = kl->w3[3 * k + a];
      tab[10 * k + 3 + a] = kl->amp3[3 * k + a];
      tab[10 * k + 6 + a] = (double)kl->idx3[3 * k + a];
    }
    tab[10 * k + 9] = kl->eig[k];
    if (!(kl->eig[k] >= 0)) return set_error(ctx, MSG_ERR_INVALID_ARGUMENT, "KL eigenvalue %d is negative", k);
  }
  // table and psi live in context workspace slots 16 and 15 (no per-call allocation)
  void *d_tab = nullptr, *d_psi = nullptr;
  MSG_TRY(workspace(ctx, 16, sizeof(double) * tab.size(), &d_tab));
  MSG_TRY(workspace(ctx, 15, sizeof(double) * (size_t)K * m->n_elems, &d_psi));
  // through the context's pinned staging buffer when there is one: a pageable
  // upload can wait behind device-to-host copies still in flight
  // (MSG_MC_SOLVE_BATCH_PIPELINED), a pinned one is a plain async copy. The
  // buffer is free again: every earlier use was followed by a stream sync.
  const double* src = tab.data();
  if (ctx->h_stage && tab.size() * sizeof(double) <= 8192) {
    MSG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    std::memcpy(ctx->h_stage, tab.data(), sizeof(double) * tab.size());
    src = ctx->h_stage;
  }
  MSG_CUDA(ctx, cudaMemcpyAsync(d_tab, src, sizeof(double) * tab.size(), cudaMemcpyHostToDevice, ctx->stream));
  dim3 grid((m->n_elems + 127) / 128, K);
  out->psi = static_cast<double*>(d_psi);
  k_kl_psi<<<grid, 128, 0, ctx->stream>>>(m->n_elems, K, m->d_centroid.as<double>(), static_cast<double*>(d_tab),
                                          kl->domain[0], kl->domain[1], kl->domain[2], kl->sigma, out->psi);
  count_launch(ctx);
  MSG_CUDA(ctx, cudaGetLastError());
  // the host table is staged synchronously by the pageable copy; nothing to wait for
  out->n_terms = K;
  out->mu = std::log(kl->mean) - (kl->mean_correction ? 0.5 * kl->sigma * kl->sigma : 0.0);
  out->gaussian = kl->gaussian ? 1 : 0;
  out->mean = kl->mean;
  return MSG_OK;
}

namespace {
__global__ void k_publish_flags(const int* __restrict__ src, int* dst, int n) {
  for (int i = threadIdx.x; i < n; i += blockDim.x) dst[i] = src[i];
}
}  // namespace

int publish_flags(Context* ctx, const int* d_src, int n, int* h_host, int* d_hmapped, cudaStream_t st) {
  if (d_hmapped && n <= 1024) {
    k_publish_flags<<<1, n <= 32 ? 32 : 256, 0, st>>>(d_src, d_hmapped, n);
    count_launch(ctx);
    MSG_CUDA(ctx, cudaGetLastError());
    return MSG_OK;
  }
  MSG_CUDA(ctx, cudaMemcpyAsync(h_host, d_src, sizeof(int) * n, cudaMemcpyDeviceToHost, st));
  return MSG_OK;
}

int launch_kl_field(Context* ctx, const Mesh* m, const KLDevice* kl, int R, int Rp, const double* d_xi,
                    double* d_E64_er, float* d_E32_er, double* d_E64_re, const int* d_elem_row) {
  dim3 grid((m->n_elems + 31) / 32, Rp / 32);
  k_kl_field<<<grid, dim3(32, 8), 0, ctx->stream>>>(m->n_elems, kl->n_terms, R, Rp, d_xi, kl->psi,
                                                    kl->mu, kl->gaussian, kl->mean, d_E64_er, d_E32_er, d_E64_re,
                                                    d_elem_row);
  count_launch(ctx);
  MSG_CUDA(ctx, cudaGetLastError());
  return MSG_OK;
}

}  // namespace msg
