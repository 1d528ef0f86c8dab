// Replays the reference's analyzer call sequences through the C++ host mirror
// (msolve.hpp) against the C ABI, and writes the results as raw little-endian
// binary for the tests:
//
//   model   cantilever|block N OUT       n_dofs (int32), DOF map [n_nodes][3] (int32), forces [n_dofs] (f64)
//   static  cantilever|block N OUT [mixed]
//           StaticAnalyzer(ProblemStructural, LinearAnalyzer(SolverPCG)):
//           BuildMatrices, Initialize, Solve(1e-10) -> iterations (int32),
//           relative residual (f64), solution [n_dofs] (f64)
//   mc      N R TERMS XI OUT [fp64]      MonteCarloAnalyzerWithStochasticMaterial on the N^3 clamped
//           block with xi [R][TERMS] read from XI (f64): tip [R], residuals [R] (f64),
//           iterations [R] (int32), solutions [R][n_dofs] (f64)
//   ragged  N1 N2 R TERMS XI OUT         RaggedMonteCarloBatch of two analyzers (the N1^3 clamped block
//           and the N2^3 one with move_interior, R realizations each, xi [2][R][TERMS] from
//           XI, tol 1e-10) -> per analyzer: tip [R], residuals [R] (f64), iterations [R]
//           (int32), solutions [R][n_dofs] (f64)
//   newmark N R TERMS XI STEPS OUT       NewmarkDynamicAnalyzer (beta 0.25, gamma 0.5, dt 0.01,
//           Rayleigh 0.01 / 0.001, ground acceleration 0.1 sin(2 pi t) in x):
//           tip history [R][STEPS] (f64), final displacements [R][n_dofs] (f64)
//   serve   N1 N2 R TERMS XI OUT          Server with two models (N1^3 and N2^3 clamped blocks, tol
//           1e-10): R requests to each, xi rows [2][R][TERMS] from XI, all submitted before
//           the first poll -> for every request in submission order: iterations (int32),
//           relative residual (f64), displacements [n_dofs] (f64)
//   reorth  B OUT                        SolverPCGReorthogonalized on the cantilever (tol 1e-10,
//           store of 400 pairs) for the 3 loads [3][n_dofs] in B, the first from zero, the
//           others from the store -> per load: iterations, stored pairs (int32), solution (f64)
//   stress  U OUT                        H8StressBatch over the cantilever's elements (E 1, nu 0.3) with
//           u [n_elems][24] from U -> strains, stresses [n][8][6], forces [n][24] (f64)
//   pc      N M P U OUT                  PolynomialChaosSolverPCGMatrixCalculator on the N^3 block with a
//           Gaussian field (corr 0.3 N, max(M,4) terms, 8 modes, mean 2, covariance 0.15):
//           y = MultiplyWithMatrix(u), u [PsiSize][n_dofs] from U (f64)
//   kl      N TERMS OUT                  the KL table of the N^3 block's provider: w [TERMS][3],
//           amp [TERMS][3] (f64), idx [TERMS][3] (int32), eig [TERMS] (f64) (host only)
//   errors                               the exception type each status code maps to, one per line
//           (host only)
//   guard                                 the Newmark coefficient guards (alpha too small)
//
// The KL provider of mc / newmark is the separable exponential kernel with
// correlation length 0.2 N and 6 one-dimensional modes per axis, mean 1,
// sigma 0.3. Exit codes: 0 ok, 2 usage, 3 InvalidOperationException,
// 4 ArgumentException, 5 other status codes, 6 I/O.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "msolve.hpp"

namespace {

bool write_all(FILE* f, const void* p, size_t bytes) { return bytes == 0 || std::fwrite(p, 1, bytes, f) == bytes; }

template <class T> bool put(FILE* f, const std::vector<T>& v) { return write_all(f, v.data(), sizeof(T) * v.size()); }

msolve::Model make_model(const std::string& kind, int n) {
  if (kind == "cantilever") return msolve::Hexa8MeshGenerator::Cantilever();
  return msolve::Hexa8MeshGenerator::ClampedBlock(n);
}

// Interior nodes of a block moved by exact binary fractions (the same bits in
// every language): node i, axis a by 0.0625 * (((7 i + 3 a) mod 5) - 2).
void move_interior(msolve::Model& m) {
  double hi = 0.0;
  for (double v : m.xyz) hi = std::max(hi, v);
  for (int i = 0; i < m.NumNodes(); ++i) {
    bool inner = true;
    for (int a = 0; a < 3; ++a) inner = inner && m.xyz[3 * i + a] > 0.5 && m.xyz[3 * i + a] < hi - 0.5;
    if (inner)
      for (int a = 0; a < 3; ++a) m.xyz[3 * i + a] += 0.0625 * (((7 * i + 3 * a) % 5) - 2);
  }
}

std::vector<double> read_doubles(const char* path, size_t count) {
  std::vector<double> v(count);
  FILE* f = std::fopen(path, "rb");
  if (!f || std::fread(v.data(), sizeof(double), count, f) != count) {
    if (f) std::fclose(f);
    throw std::runtime_error(std::string("cannot read ") + path);
  }
  std::fclose(f);
  return v;
}

int run(int argc, char** argv) {
  if (argc < 2) return 2;
  const std::string cmd = argv[1];
  if (cmd == "model" && argc >= 5) {
    msolve::Model m = make_model(argv[2], std::atoi(argv[3]));
    FILE* f = std::fopen(argv[4], "wb");
    if (!f) return 6;
    const int32_t nd = m.n_dofs;
    const bool ok = write_all(f, &nd, sizeof(nd)) && put(f, m.dof) && put(f, m.subdomain.Forces);
    std::fclose(f);
    return ok ? 0 : 6;
  }
  if (cmd == "static" && argc >= 5) {
    msolve::Model m = make_model(argv[2], std::atoi(argv[3]));
    const bool mixed = argc >= 6 && std::string(argv[5]) == "mixed";
    msolve::Context ctx(0);
    msolve::ProblemStructural provider(ctx, m);
    msolve::SolverPCG solver(ctx, m, 20000, 1e-10, mixed);
    msolve::LinearAnalyzer child(solver);
    msolve::StaticAnalyzer parent(provider, child);
    parent.BuildMatrices();
    parent.Initialize();
    parent.Solve();
    FILE* f = std::fopen(argv[4], "wb");
    if (!f) return 6;
    const int32_t it = solver.Iterations;
    const double rr = solver.RelativeResidual;
    const bool ok = write_all(f, &it, sizeof(it)) && write_all(f, &rr, sizeof(rr)) && put(f, m.subdomain.Solution);
    std::fclose(f);
    return ok ? 0 : 6;
  }
  if (cmd == "mc" && argc >= 7) {
    const int n = std::atoi(argv[2]), R = std::atoi(argv[3]), terms = std::atoi(argv[4]);
    const bool fp64 = argc >= 8 && std::string(argv[7]) == "fp64";
    msolve::Model m = msolve::Hexa8MeshGenerator::ClampedBlock(n);
    msolve::Context ctx(0);
    msolve::LognormalStochasticCoefficientsProvider kl({(double)n, (double)n, (double)n}, 0.2 * n, terms, 6);
    msolve::MonteCarloAnalyzerWithStochasticMaterial mc(ctx, m, kl, terms, R, !fp64, 1e-10);
    mc.RandomNumbers = read_doubles(argv[5], (size_t)R * terms);
    mc.Solve();
    FILE* f = std::fopen(argv[6], "wb");
    if (!f) return 6;
    const bool ok = put(f, mc.TipValues) && put(f, mc.Residuals) && put(f, mc.Iterations) && put(f, mc.Solutions);
    std::fclose(f);
    return ok ? 0 : 6;
  }
  if (cmd == "ragged" && argc >= 8) {
    const int n1 = std::atoi(argv[2]), n2 = std::atoi(argv[3]), R = std::atoi(argv[4]), terms = std::atoi(argv[5]);
    const std::vector<double> xi = read_doubles(argv[6], (size_t)2 * R * terms);
    msolve::Context ctx(0);
    msolve::Model m1 = msolve::Hexa8MeshGenerator::ClampedBlock(n1), m2 = msolve::Hexa8MeshGenerator::ClampedBlock(n2);
    move_interior(m2);
    msolve::LognormalStochasticCoefficientsProvider k1({(double)n1, (double)n1, (double)n1}, 0.2 * n1, terms, 6);
    msolve::LognormalStochasticCoefficientsProvider k2({(double)n2, (double)n2, (double)n2}, 0.2 * n2, terms, 6);
    msolve::MonteCarloAnalyzerWithStochasticMaterial a1(ctx, m1, k1, terms, R), a2(ctx, m2, k2, terms, R);
    a1.RandomNumbers.assign(xi.begin(), xi.begin() + (size_t)R * terms);
    a2.RandomNumbers.assign(xi.begin() + (size_t)R * terms, xi.end());
    msolve::RaggedMonteCarloBatch batch(ctx, 1e-10);
    batch.Add(a1);
    batch.Add(a2);
    batch.Solve();
    FILE* f = std::fopen(argv[7], "wb");
    if (!f) return 6;
    bool ok = true;
    for (const auto* a : {&a1, &a2})
      ok = ok && put(f, a->TipValues) && put(f, a->Residuals) && put(f, a->Iterations) && put(f, a->Solutions);
    std::fclose(f);
    return ok ? 0 : 6;
  }
  if (cmd == "newmark" && argc >= 8) {
    const int n = std::atoi(argv[2]), R = std::atoi(argv[3]), terms = std::atoi(argv[4]), steps = std::atoi(argv[6]);
    msolve::Model m = msolve::Hexa8MeshGenerator::ClampedBlock(n);
    msolve::Context ctx(0);
    msolve::LognormalStochasticCoefficientsProvider kl({(double)n, (double)n, (double)n}, 0.2 * n, terms, 6);
    const double dt = 0.01;
    msolve::MassAccelerationSinusoidalLoad load{1.0, dt, dt * steps, 0.1, msolve::DOFType::X};
    msolve::NewmarkDynamicAnalyzer nm(ctx, m, kl, 0.25, 0.5, dt, dt * steps, load, R, 1.0, 0.01, 0.001, 1e-10);
    nm.RandomNumbers = read_doubles(argv[5], (size_t)R * terms);
    nm.BuildMatrices();
    nm.Solve();
    FILE* f = std::fopen(argv[7], "wb");
    if (!f) return 6;
    const bool ok = put(f, nm.TipHistory) && put(f, nm.Solutions);
    std::fclose(f);
    return ok ? 0 : 6;
  }
  if (cmd == "serve" && argc >= 8) {
    const int n1 = std::atoi(argv[2]), n2 = std::atoi(argv[3]), R = std::atoi(argv[4]), terms = std::atoi(argv[5]);
    msolve::Model m1 = msolve::Hexa8MeshGenerator::ClampedBlock(n1);
    msolve::Model m2 = msolve::Hexa8MeshGenerator::ClampedBlock(n2);
    msolve::Context ctx(0);
    msolve::LognormalStochasticCoefficientsProvider kl1({(double)n1, (double)n1, (double)n1}, 0.2 * n1, terms, 6);
    msolve::LognormalStochasticCoefficientsProvider kl2({(double)n2, (double)n2, (double)n2}, 0.2 * n2, terms, 6);
    const std::vector<double> xi = read_doubles(argv[6], (size_t)2 * R * terms);
    msolve::Server srv(ctx, 32);
    const int id[2] = {srv.AddModel(m1, kl1, 1e-10), srv.AddModel(m2, kl2, 1e-10)};
    std::vector<MSG_REQ> reqs;
    for (int k = 0; k < 2; ++k)
      for (int r = 0; r < R; ++r)
        reqs.push_back(srv.Submit(id[k], std::vector<double>(xi.begin() + ((size_t)k * R + r) * terms,
                                                             xi.begin() + ((size_t)k * R + r + 1) * terms)));
    FILE* f = std::fopen(argv[7], "wb");
    if (!f) return 6;
    bool ok = true;
    for (MSG_REQ q : reqs) {
      const msolve::Server::Result res = srv.Poll(q, -1);
      const int32_t it = res.Iterations;
      ok = ok && write_all(f, &it, sizeof(it)) && write_all(f, &res.RelativeResidual, sizeof(double)) &&
           put(f, res.X);
    }
    std::fclose(f);
    return ok ? 0 : 6;
  }
  if (cmd == "reorth" && argc >= 4) {
    msolve::Model m = msolve::Hexa8MeshGenerator::Cantilever();
    msolve::Context ctx(0);
    msolve::ProblemStructural provider(ctx, m);
    msolve::GpuMatrix& K = provider.CalculateMatrix(m.subdomain);
    msolve::SolverPCGReorthogonalizationSearchVectorCalculator search(provider.Mesh(), 400);
    msolve::SolverPCGReorthogonalized solver(ctx, m, search, 20000, 1e-10);
    solver.Matrix = &K;
    solver.Initialize();
    const std::vector<double> b = read_doubles(argv[2], (size_t)3 * m.n_dofs);
    FILE* f = std::fopen(argv[3], "wb");
    if (!f) return 6;
    bool ok = true;
    for (int k = 0; k < 3; ++k) {
      m.subdomain.Forces.assign(b.begin() + (size_t)k * m.n_dofs, b.begin() + (size_t)(k + 1) * m.n_dofs);
      solver.StartFromStore = k == 0 ? 0 : 1;
      solver.Solve();
      const int32_t hdr[2] = {solver.Iterations, search.Count()};
      ok = ok && write_all(f, hdr, sizeof(hdr)) && put(f, m.subdomain.Solution);
    }
    std::fclose(f);
    return ok ? 0 : 6;
  }
  if (cmd == "stress" && argc >= 4) {
    msolve::Model m = msolve::Hexa8MeshGenerator::Cantilever();
    msolve::Context ctx(0);
    const int ne = m.NumElements();
    std::vector<double> xyz((size_t)ne * 24);
    for (int e = 0; e < ne; ++e)
      for (int a = 0; a < 8; ++a)
        for (int c = 0; c < 3; ++c) xyz[((size_t)e * 8 + a) * 3 + c] = m.xyz[(size_t)m.conn[(size_t)e * 8 + a] * 3 + c];
    const std::vector<double> u = read_doubles(argv[2], (size_t)ne * 24);
    std::vector<double> eps, sig, frc;
    msolve::H8StressBatch(ctx, xyz, m.E_elem, m.Poisson, u, {}, eps, sig, frc);
    FILE* f = std::fopen(argv[3], "wb");
    if (!f) return 6;
    const bool ok = put(f, eps) && put(f, sig) && put(f, frc);
    std::fclose(f);
    return ok ? 0 : 6;
  }
  if (cmd == "pc" && argc >= 7) {
    const int n = std::atoi(argv[2]), mv = std::atoi(argv[3]), pd = std::atoi(argv[4]);
    msolve::Model m = msolve::Hexa8MeshGenerator::ClampedBlock(n);
    msolve::Context ctx(0);
    msolve::GaussianStochasticCoefficientsProvider kl({(double)n, (double)n, (double)n}, 0.3 * n, std::max(mv, 4), 8,
                                                      2.0, 0.15);
    msolve::GpuMesh mesh(ctx, m);
    msolve::PolynomialChaosSolverPCGMatrixCalculator op(mesh, kl, mv, pd);
    const std::vector<double> u = read_doubles(argv[5], (size_t)op.PsiSize() * m.n_dofs);
    const std::vector<double> y = op.MultiplyWithMatrix(u);
    FILE* f = std::fopen(argv[6], "wb");
    if (!f) return 6;
    const bool ok = put(f, y);
    std::fclose(f);
    return ok ? 0 : 6;
  }
  if (cmd == "kl" && argc >= 5) {
    const int n = std::atoi(argv[2]), terms = std::atoi(argv[3]);
    msolve::LognormalStochasticCoefficientsProvider kl({(double)n, (double)n, (double)n}, 0.2 * n, terms, 6);
    FILE* f = std::fopen(argv[4], "wb");
    if (!f) return 6;
    const bool ok = put(f, kl.W()) && put(f, kl.Amp()) && put(f, kl.Idx()) && put(f, kl.Eig());
    std::fclose(f);
    return ok ? 0 : 6;
  }
  if (cmd == "errors") {
    const int codes[] = {MSG_ERR_NOT_CONVERGED, MSG_ERR_BREAKDOWN, MSG_ERR_NEG_DET, MSG_ERR_NOT_STRUCTURED,
                         MSG_ERR_INVALID_ARGUMENT, MSG_ERR_OUT_OF_MEMORY, MSG_ERR_TIMEOUT, MSG_ERR_CUDA};
    for (int c : codes) {
      const char* kind = "none";
      try {
        msolve::Check(c, nullptr, "status");
      } catch (const msolve::InvalidOperationException&) {
        kind = "InvalidOperationException";
      } catch (const msolve::ArgumentException&) {
        kind = "ArgumentException";
      } catch (const msolve::MSolveException& e) {
        kind = e.Code == c ? "MSolveException" : "wrong-code";
      }
      std::printf("%d %s\n", c, kind);
    }
    return 0;
  }
  if (cmd == "guard") {
    msolve::Model m = msolve::Hexa8MeshGenerator::ClampedBlock(2);
    msolve::Context ctx(0);
    msolve::LognormalStochasticCoefficientsProvider kl({2.0, 2.0, 2.0}, 0.4, 4, 4);
    msolve::MassAccelerationSinusoidalLoad load{1.0, 0.01, 0.1, 0.1, msolve::DOFType::X};
    msolve::NewmarkDynamicAnalyzer nm(ctx, m, kl, 0.1, 0.5, 0.01, 0.1, load, 1);
    nm.BuildMatrices();  // alpha 0.1 < 0.25: InvalidOperationException
    return 0;
  }
  return 2;
}

}  // namespace

int main(int argc, char** argv) {
  try {
    const int rc = run(argc, argv);
    if (rc == 2) std::fprintf(stderr, "usage: see the header of msolve_driver.cpp\n");
    return rc;
  } catch (const msolve::InvalidOperationException& e) {
    std::fprintf(stderr, "InvalidOperationException: %s\n", e.what());
    return 3;
  } catch (const msolve::ArgumentException& e) {
    std::fprintf(stderr, "ArgumentException: %s\n", e.what());
    return 4;
  } catch (const msolve::MSolveException& e) {
    std::fprintf(stderr, "MSolveException: %s\n", e.what());
    return 5;
  } catch (const std::exception& e) {
    std::fprintf(stderr, "error: %s\n", e.what());
    return 6;
  }
}
