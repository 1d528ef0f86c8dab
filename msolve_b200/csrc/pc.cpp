// Polynomial-chaos Galerkin coefficients for Gaussian germs, the host twin of
// PolynomialChaosCoefficientsCalculator
// (ISAAR.MSolve.PreProcessor/Stochastic/PolynomialChaosCoefficientsCalculator.cs:30-456,
// Gaussian branch): the multi-index basis of m variables up to total degree p
// in the reference's enumeration order, the squared norms prod_l (alpha_l)!,
// and for every output block j the terms (matrix pos, input block k, weight)
// of  y_j = sum_pos sum_k c K_pos u_k  (MultiplyWithMatrix,
// PolynomialChaosSolverPCGMatrixCalculator.cs:1062-1089): pos 0 couples j with
// itself by <psi_j^2>; pos i+1 couples blocks whose indices differ only in
// variable i, by one, with <xi_i psi_j psi_k> (Hermite recurrence).
#include <tuple>

#include "msg_internal.h"

namespace msg {

namespace {
double factorial(int f) {
  double r = 1;
  for (int i = 2; i <= f; ++i) r *= i;
  return r;
}
}  // namespace

int pc_size(int m, int p) {
  if (m < 1 || p < 1) return -1;
  double s = 0;
  for (int k = 0; k <= p; ++k) s += factorial(m + k - 1) / (factorial(k) * factorial(m - 1));
  return (int)s;
}

int pc_basis(int m, int p, std::vector<int>& basis, std::vector<int>& norms) {
  const int P = pc_size(m, p);
  if (P < 0) return MSG_ERR_INVALID_ARGUMENT;
  basis.assign((size_t)P * m, 0);
  auto B = [&](int n, int l) -> int& { return basis[(size_t)n * m + l]; };
  if (m == 1) {
    // the reference fills index i (not i + 1) for the one-variable case; kept as it is
    for (int i = 0; i < p; ++i) B(i + 1, 0) = i;
  } else {
    // compositions of each total degree d into m parts, generated as increasing
    // bar positions t[0..m-2] in 1..m-1+d (the reference's order)
    const int nb = m - 1;
    std::vector<int> t(nb);
    int n = 0;
    for (int d = 1; d <= p; ++d) {
      bool started = false, done = false;
      while (!done) {
        ++n;
        if (!started) {
          for (int i = 0; i < nb; ++i) t[i] = i + 1;
          started = true;
        } else if (t[nb - 1] < nb + d) {
          t[nb - 1] += 1;
        } else {
          int j = nb;
          while (t[j - 1] == j + d) --j;
          t[j - 1] += 1;
          for (int k = j; k < nb; ++k) t[k] = t[j - 1] + k - j + 1;
        }
        B(n, 0) = t[0] - 1;
        for (int i = 1; i < nb; ++i) B(n, i) = t[i] - t[i - 1] - 1;
        B(n, nb) = m + d - t[nb - 1] - 1;
        if (t[0] == d + 1) done = true;
      }
    }
  }
  norms.assign(P, 1);
  for (int k = 0; k < P; ++k) {
    int nn = 1;
    for (int l = 0; l < m; ++l) nn *= (int)factorial(B(k, l));
    norms[k] = nn;
  }
  return MSG_OK;
}

int pc_gaussian_terms(int m, int p, std::vector<int>& term_ptr, std::vector<int>& term_pos,
                      std::vector<int>& term_k, std::vector<double>& term_c) {
  std::vector<int> basis, norms;
  MSG_TRY(pc_basis(m, p, basis, norms));
  const int P = (int)norms.size();
  auto B = [&](int n, int l) { return basis[(size_t)n * m + l]; };
  // the reference's lists per matrix: pos 0 diagonal, pos i+1 nearest neighbours in variable i
  std::vector<std::vector<std::tuple<int, int, double>>> by_row(P);
  for (int j = 0; j < P; ++j) by_row[j].emplace_back(0, j, (double)norms[j]);
  for (int i = 0; i < m; ++i)
    for (int j = 0; j < P; ++j)
      for (int k = 0; k < P; ++k) {
        bool other = false;
        for (int l = 0; l < m && !other; ++l)
          if (l != i && B(j, l) != B(k, l)) other = true;
        if (other) continue;
        if (B(k, i) == B(j, i) - 1)
          by_row[j].emplace_back(i + 1, k, (double)norms[j]);
        else if (B(k, i) == B(j, i) + 1)
          by_row[j].emplace_back(i + 1, k, (double)norms[j] * (B(j, i) + 1));
      }
  term_ptr.assign(P + 1, 0);
  term_pos.clear();
  term_k.clear();
  term_c.clear();
  for (int j = 0; j < P; ++j) {
    for (const auto& t : by_row[j]) {
      term_pos.push_back(std::get<0>(t));
      term_k.push_back(std::get<1>(t));
      term_c.push_back(std::get<2>(t));
    }
    term_ptr[j + 1] = (int)term_pos.size();
  }
  return MSG_OK;
}

}  // namespace msg
