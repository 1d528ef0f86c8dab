// C++ host-side mirror of the reference's preprocessor, provider, solver and
// analyzer interfaces over the C ABI of include/msolve_gpu.h (header-only,
// C++17). The reference is C# (.NET 4) calling native code through P/Invoke;
// this layer keeps its class names, call sequence and error behaviour so a
// C++ host (or a C# shim written after it) drives the GPU path the way
// StaticAnalyzer / MonteCarloAnalyzerWithStochasticMaterial drive skyline
// solvers in the reference:
//
//   msolve::Model model = msolve::Hexa8MeshGenerator::Cantilever();
//   msolve::Context ctx(0);
//   msolve::ProblemStructural provider(ctx, model);              // IStaticProvider
//   msolve::SolverPCG solver(ctx, model);                        // ISolver
//   msolve::LinearAnalyzer child(solver);                        // IAnalyzer
//   msolve::StaticAnalyzer parent(provider, child);              // IAnalyzer
//   parent.BuildMatrices(); parent.Initialize(); parent.Solve();
//   model.subdomain.Solution ...
//
// References (project paths): Model.cs:165-238 (EnumerateGlobalDOFs,
// AssignNodalLoads), Hexa8MeshGenerator.cs:508-568,1075-1089 (node and element
// order), ProblemStructural.cs:63-89,217-221, SolverPCGSkyline.cs:75-108,
// SolverPCG.cs:105-149, LinearAnalyzer.cs:12-69, StaticAnalyzer.cs:10-75,
// LognormalFileStochasticCoefficientsProvider.cs:43-193,
// MonteCarloAnalyzerWithStochasticMaterial.cs:55-296,
// NewmarkDynamicAnalyzer.cs:16-315, MassAccelerationSinusoidalLoad.cs:11-31.
// Status codes map to the exception types the reference throws
// (InvalidOperationException, ArgumentException).
#pragma once

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <memory>
#include <random>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "msolve_gpu.h"

namespace msolve {

// ------------------------------------------------------------------ errors
class MSolveException : public std::runtime_error {
 public:
  MSolveException(int code, const std::string& msg)
      : std::runtime_error("[" + std::to_string(code) + "] " + msg), Code(code) {}
  int Code;
};
class InvalidOperationException : public MSolveException {
  using MSolveException::MSolveException;
};
class ArgumentException : public MSolveException {
  using MSolveException::MSolveException;
};

inline void Check(int status, MSG_CTX ctx, const std::string& what) {
  if (status == MSG_OK) return;
  std::string msg = what;
  if (ctx) {
    const char* e = MSG_LAST_ERROR(ctx);
    if (e && *e) msg += std::string(": ") + e;
  }
  if (status == MSG_ERR_INVALID_ARGUMENT) throw ArgumentException(status, msg);
  if (status == MSG_ERR_NOT_CONVERGED || status == MSG_ERR_BREAKDOWN || status == MSG_ERR_NEG_DET ||
      status == MSG_ERR_NOT_STRUCTURED)
    throw InvalidOperationException(status, msg);
  throw MSolveException(status, msg);
}

// ------------------------------------------------------------------ model
enum class DOFType : int { X = 0, Y = 1, Z = 2 };

// ISolverSubdomain analogue: the right-hand side (Forces) and the Solution of
// the single subdomain of a model.
struct Subdomain {
  int ID = 1;
  std::vector<double> Forces;
  std::vector<double> Solution;
  const std::vector<double>& RHS() const { return Forces; }
};

// Nodes (x fastest in generator order), Hexa8 elements (bottom face counter-
// clockwise, then top), constraints, nodal loads, material.
class Model {
 public:
  std::vector<double> xyz;                    // [n_nodes][3]
  std::vector<int> conn;                      // [n_elems][8]
  std::vector<std::array<bool, 3>> constraints;
  struct Load {
    int node;
    DOFType dof;
    double amount;
  };
  std::vector<Load> loads;
  double Young = 1.0, Poisson = 0.3, Density = 1.0;
  std::vector<double> E_elem;                 // per-element modulus of the static path
  std::vector<int> dof;                       // [n_nodes][3], -1 constrained
  int n_dofs = 0;
  Subdomain subdomain;
  bool structured = false;
  int nx = 0, ny = 0, nz = 0;
  double h = 1.0;

  int NumNodes() const { return (int)(xyz.size() / 3); }
  int NumElements() const { return (int)(conn.size() / 8); }
  void Constrain(int node) { constraints[node] = {true, true, true}; }
  void AddLoad(int node, DOFType d, double amount) { loads.push_back({node, d, amount}); }

  // Model.EnumerateGlobalDOFs (ascending node, X, Y, Z, constrained -> -1) and
  // Model.AssignNodalLoads (assignment per DOF, not accumulation: :236).
  Model& ConnectDataStructures() {
    const int nn = NumNodes();
    dof.assign((size_t)nn * 3, -1);
    int k = 0;
    for (int n = 0; n < nn; ++n)
      for (int c = 0; c < 3; ++c)
        if (!constraints[n][c]) dof[(size_t)n * 3 + c] = k++;
    n_dofs = k;
    subdomain.Forces.assign(n_dofs, 0.0);
    for (const Load& l : loads) {
      const int d = dof[(size_t)l.node * 3 + (int)l.dof];
      if (d >= 0) subdomain.Forces[d] = l.amount;
    }
    return *this;
  }
  int DofOf(int node, DOFType d) const { return dof[(size_t)node * 3 + (int)d]; }
};

// Structured blocks of equal cubes in the reference generator's order.
struct Hexa8MeshGenerator {
  static bool Close(double a, double b) { return std::fabs(a - b) <= 1e-8 + 1e-5 * std::fabs(b); }

  static Model Block(int nx, int ny, int nz, double h = 1.0, double young = 1.0, double poisson = 0.3,
                     double density = 1.0) {
    Model m;
    m.Young = young;
    m.Poisson = poisson;
    m.Density = density;
    const int NX = nx + 1, NXY = (nx + 1) * (ny + 1);
    for (int k = 0; k <= nz; ++k)
      for (int j = 0; j <= ny; ++j)
        for (int i = 0; i <= nx; ++i) {
          m.xyz.push_back(i * h);
          m.xyz.push_back(j * h);
          m.xyz.push_back(k * h);
        }
    for (int k = 0; k < nz; ++k)
      for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
          const int b = i + NX * j + NXY * k;
          const int c[8] = {b, b + 1, b + NX + 1, b + NX, b + NXY, b + NXY + 1, b + NXY + NX + 1, b + NXY + NX};
          m.conn.insert(m.conn.end(), c, c + 8);
        }
    m.constraints.assign(m.NumNodes(), {false, false, false});
    m.E_elem.assign(m.NumElements(), young);
    m.structured = true;
    m.nx = nx;
    m.ny = ny;
    m.nz = nz;
    m.h = h;
    return m;
  }
  static std::vector<int> ClampPlane(Model& m, int axis, double value = 0.0) {
    std::vector<int> nodes;
    for (int n = 0; n < m.NumNodes(); ++n)
      if (Close(m.xyz[(size_t)n * 3 + axis], value)) {
        m.Constrain(n);
        nodes.push_back(n);
      }
    return nodes;
  }
  static double AxisMax(const Model& m, int axis) {
    double v = -1e300;
    for (int n = 0; n < m.NumNodes(); ++n) v = std::max(v, m.xyz[(size_t)n * 3 + axis]);
    return v;
  }
  // total load in `direction`, split equally over the nodes of the face at the maximum of `axis`
  static void TipLoad(Model& m, int axis, DOFType direction, double total) {
    const double mx = AxisMax(m, axis);
    std::vector<int> face;
    for (int n = 0; n < m.NumNodes(); ++n)
      if (Close(m.xyz[(size_t)n * 3 + axis], mx)) face.push_back(n);
    for (int n : face) m.AddLoad(n, direction, total / (double)face.size());
  }
  // uniform pressure p in -z on the top face, consistent bilinear weights
  // (interior 1, edge 1/2, corner 1/4 of p h^2)
  static void TopPressure(Model& m, double p = 1.0) {
    const double zmax = AxisMax(m, 2);
    for (int n = 0; n < m.NumNodes(); ++n) {
      if (!Close(m.xyz[(size_t)n * 3 + 2], zmax)) continue;
      const double xs = m.xyz[(size_t)n * 3] / m.h, ys = m.xyz[(size_t)n * 3 + 1] / m.h;
      const int cx = (Close(xs, 0.0) || Close(xs, (double)m.nx)) ? 1 : 2;
      const int cy = (Close(ys, 0.0) || Close(ys, (double)m.ny)) ? 1 : 2;
      m.AddLoad(n, DOFType::Z, -p * m.h * m.h * cx * cy / 4.0);
    }
  }
  // 10 x 4 x 4 cantilever: x = 0 clamped, total -1 in z over the x = max face
  static Model Cantilever(int nx = 10, int ny = 4, int nz = 4, double young = 1.0, double poisson = 0.3,
                          double total = -1.0) {
    Model m = Block(nx, ny, nz, 1.0, young, poisson);
    ClampPlane(m, 0, 0.0);
    TipLoad(m, 0, DOFType::Z, total);
    return m.ConnectDataStructures(), m;
  }
  // n^3 block, z = 0 clamped, unit pressure on the top face
  static Model ClampedBlock(int n, double young = 1.0, double poisson = 0.3, double p = 1.0) {
    Model m = Block(n, n, n, 1.0, young, poisson);
    ClampPlane(m, 2, 0.0);
    TopPressure(m, p);
    return m.ConnectDataStructures(), m;
  }
  // u_z of the node at the far corner (max x, then y, then z)
  static int TipDof(const Model& m) {
    int best = 0;
    double bv = -1e300;
    for (int n = 0; n < m.NumNodes(); ++n) {
      const double v = m.xyz[(size_t)n * 3] + m.xyz[(size_t)n * 3 + 1] * 1e3 + m.xyz[(size_t)n * 3 + 2] * 1e6;
      if (v > bv) {
        bv = v;
        best = n;
      }
    }
    return m.DofOf(best, DOFType::Z);
  }
};

// ------------------------------------------------------------------ device handles
class Context {
 public:
  explicit Context(int device = 0, uint64_t mem_budget_bytes = 0) : device_(device) {
    Check(MSG_CREATE(device, mem_budget_bytes, &h_), nullptr, "MSG_CREATE");
  }
  ~Context() {
    if (h_) MSG_DESTROY(h_);
  }
  Context(const Context&) = delete;
  Context& operator=(const Context&) = delete;
  MSG_CTX Handle() const { return h_; }
  void SetOption(const char* key, double value) { Check(MSG_SET_OPTION(h_, key, value), h_, "MSG_SET_OPTION"); }
  double GetOption(const char* key) const {
    double v = 0.0;
    Check(MSG_GET_OPTION(h_, key, &v), h_, "MSG_GET_OPTION");
    return v;
  }

 private:
  MSG_CTX h_ = nullptr;
  int device_;
};

class GpuMesh {
 public:
  GpuMesh(Context& ctx, Model& model) : ctx_(ctx), model_(model) {
    if (model.dof.empty()) model.ConnectDataStructures();
    Check(MSG_MESH_CREATE(ctx.Handle(), model.NumNodes(), model.xyz.data(), model.NumElements(), model.conn.data(),
                          model.dof.data(), model.n_dofs, &h_),
          ctx.Handle(), "MSG_MESH_CREATE");
  }
  ~GpuMesh() {
    if (h_) MSG_MESH_DESTROY(h_);
  }
  GpuMesh(const GpuMesh&) = delete;
  GpuMesh& operator=(const GpuMesh&) = delete;
  MSG_MESH Handle() const { return h_; }
  Context& Ctx() const { return ctx_; }
  Model& GetModel() const { return model_; }

 private:
  Context& ctx_;
  Model& model_;
  MSG_MESH h_ = nullptr;
};

// IMatrix2D analogue: the assembled global stiffness on the device.
class GpuMatrix {
 public:
  GpuMatrix(GpuMesh& mesh, const std::vector<double>& E, double nu) : mesh_(mesh) {
    Check(MSG_ASSEMBLE_BSR(mesh.Handle(), E.data(), nu, &h_), mesh.Ctx().Handle(), "MSG_ASSEMBLE_BSR");
  }
  ~GpuMatrix() {
    if (h_) MSG_MAT_DESTROY(h_);
  }
  GpuMatrix(const GpuMatrix&) = delete;
  GpuMatrix& operator=(const GpuMatrix&) = delete;
  MSG_MAT Handle() const { return h_; }
  std::vector<double> Multiply(const std::vector<double>& x) const {
    std::vector<double> y(mesh_.GetModel().n_dofs);
    Check(MSG_MAT_MULTIPLY(h_, x.data(), y.data()), mesh_.Ctx().Handle(), "Multiply");
    return y;
  }

 private:
  GpuMesh& mesh_;
  MSG_MAT h_ = nullptr;
};

// ------------------------------------------------------------------ providers, solvers, analyzers
// IStaticProvider: ProblemStructural.BuildKs / CalculateMatrix on the device.
class ProblemStructural {
 public:
  ProblemStructural(Context& ctx, Model& model) : model_(model), mesh_(ctx, model) {}
  GpuMatrix& CalculateMatrix(Subdomain&) {
    if (!K_) K_.reset(new GpuMatrix(mesh_, model_.E_elem, model_.Poisson));
    return *K_;
  }
  void Reset() { K_.reset(); }
  Model& GetModel() { return model_; }
  GpuMesh& Mesh() { return mesh_; }

 private:
  Model& model_;
  GpuMesh mesh_;
  std::unique_ptr<GpuMatrix> K_;
};

class ISolver {
 public:
  virtual ~ISolver() = default;
  virtual void Initialize() = 0;
  virtual void Solve() = 0;
};

// SolverPCG<T> over the device Jacobi-PCG. Solve() uses (20000, 1e-7) as
// SolverPCG<T>.Solve() does; precision "mixed": FP32 matrix values in the
// loop with FP64 refinement to the FP64 true residual.
class SolverPCG : public ISolver {
 public:
  SolverPCG(Context& ctx, Model& model, int max_iterations = 20000, double tolerance = 1e-7, bool mixed = false)
      : ctx_(ctx), model_(model), MaxIterations(max_iterations), Tolerance(tolerance), Mixed(mixed) {}
  void Initialize() override {
    if (!Matrix) throw InvalidOperationException(MSG_ERR_INVALID_ARGUMENT, "no matrix: call BuildMatrices first");
  }
  void Solve() override {
    Subdomain& s = model_.subdomain;
    s.Solution.assign(model_.n_dofs, 0.0);
    int it = 0;
    double rr = 0.0;
    const int st = (Mixed ? MSG_PCG_SOLVE_MIXED : MSG_PCG_SOLVE)(Matrix->Handle(), s.Forces.data(), s.Solution.data(),
                                                                 MaxIterations, Tolerance, &it, &rr);
    Iterations = it;
    RelativeResidual = rr;
    Check(st, ctx_.Handle(), "MSG_PCG_SOLVE");
  }
  GpuMatrix* Matrix = nullptr;
  int Iterations = 0;
  double RelativeResidual = 0.0;

 protected:
  Context& ctx_;
  Model& model_;

 public:
  int MaxIterations;
  double Tolerance;
  bool Mixed;
};

class IAnalyzer {
 public:
  virtual ~IAnalyzer() = default;
  virtual void BuildMatrices() {}
  virtual void Initialize() = 0;
  virtual void Solve() = 0;
  IAnalyzer* ParentAnalyzer = nullptr;
};

class LinearAnalyzer : public IAnalyzer {
 public:
  explicit LinearAnalyzer(SolverPCG& solver) : solver_(solver) {}
  void Initialize() override { solver_.Initialize(); }
  void Solve() override { solver_.Solve(); }
  SolverPCG& Solver() { return solver_; }

 private:
  SolverPCG& solver_;
};

class StaticAnalyzer : public IAnalyzer {
 public:
  StaticAnalyzer(ProblemStructural& provider, LinearAnalyzer& child) : provider_(provider), child_(child) {
    child.ParentAnalyzer = this;
  }
  void BuildMatrices() override {
    child_.Solver().Matrix = &provider_.CalculateMatrix(provider_.GetModel().subdomain);
  }
  void Initialize() override { child_.Initialize(); }
  void Solve() override { child_.Solve(); }

 private:
  ProblemStructural& provider_;
  LinearAnalyzer& child_;
};

// KL lognormal Young's modulus with the analytic table of the separable
// exponential kernel (the reference reads the same table from a file).
class LognormalStochasticCoefficientsProvider {
 public:
  LognormalStochasticCoefficientsProvider(std::array<double, 3> domain, double corr_len, int n_terms = 50,
                                          int n1d = 16, double mean = 1.0, double sigma = 0.3,
                                          bool mean_correction = false)
      : domain_(domain), w_(3 * n_terms), amp_(3 * n_terms), idx_(3 * n_terms), eig_(n_terms) {
    kl_ = MSG_KL{};
    Check(MSG_KL_TABLE(domain_.data(), corr_len, n_terms, n1d, w_.data(), amp_.data(), idx_.data(), eig_.data()),
          nullptr, "MSG_KL_TABLE");
    kl_.n_terms = n_terms;
    kl_.w3 = w_.data();
    kl_.amp3 = amp_.data();
    kl_.idx3 = idx_.data();
    kl_.eig = eig_.data();
    for (int a = 0; a < 3; ++a) kl_.domain[a] = domain_[a];
    kl_.mean = mean;
    kl_.sigma = sigma;
    kl_.mean_correction = mean_correction ? 1 : 0;
    kl_.gaussian = 0;
  }
  LognormalStochasticCoefficientsProvider(const LognormalStochasticCoefficientsProvider&) = delete;
  LognormalStochasticCoefficientsProvider& operator=(const LognormalStochasticCoefficientsProvider&) = delete;
  const MSG_KL* Kl() const { return &kl_; }
  int Terms() const { return kl_.n_terms; }
  bool Gaussian() const { return kl_.gaussian != 0; }
  const std::vector<double>& W() const { return w_; }
  const std::vector<double>& Amp() const { return amp_; }
  const std::vector<int>& Idx() const { return idx_; }
  const std::vector<double>& Eig() const { return eig_; }

 private:
  std::array<double, 3> domain_;
  std::vector<double> w_, amp_;
  std::vector<int> idx_;
  std::vector<double> eig_;

 protected:
  MSG_KL kl_;
};

// KL Gaussian modulus E = mean (1 + sum_k xi_k covariance sqrt(eig_k) phi_k)
// (GaussianFileStochasticCoefficientsProvider.cs:24-108; covariance 0.15 as the reference).
class GaussianStochasticCoefficientsProvider : public LognormalStochasticCoefficientsProvider {
 public:
  GaussianStochasticCoefficientsProvider(std::array<double, 3> domain, double corr_len, int n_terms = 50,
                                         int n1d = 16, double mean = 1.0, double covariance = 0.15)
      : LognormalStochasticCoefficientsProvider(domain, corr_len, n_terms, n1d, mean, covariance) {
    kl_.gaussian = 1;
  }
};

// The realization loop: Initialize() draws xi[simulations][expansionOrder] ~
// N(0, 1) (the reference's random stream is outside parity; a caller may set
// RandomNumbers itself), Solve() runs every realization through
// MSG_MC_SOLVE_BATCH (batched mixed precision, or the FP64 drop-in one
// realization after another).
class MonteCarloAnalyzerWithStochasticMaterial : public IAnalyzer {
 public:
  MonteCarloAnalyzerWithStochasticMaterial(Context& ctx, Model& model,
                                           LognormalStochasticCoefficientsProvider& provider, int expansion_order,
                                           int simulations, bool mixed = true, double tolerance = 1e-8,
                                           int max_iterations = 20000, uint64_t seed = 12345)
      : ctx_(ctx), model_(model), kl_(provider), mesh_(ctx, model), expansionOrder_(expansion_order),
        simulations_(simulations), Mixed(mixed), Tolerance(tolerance), MaxIterations(max_iterations), seed_(seed) {
    if (expansion_order != provider.Terms())
      throw ArgumentException(MSG_ERR_INVALID_ARGUMENT, "expansion order differs from the provider's terms");
    TipDof = Hexa8MeshGenerator::TipDof(model);
  }
  void Initialize() override {
    std::mt19937_64 rng(seed_);
    std::normal_distribution<double> n01(0.0, 1.0);
    RandomNumbers.resize((size_t)simulations_ * expansionOrder_);
    for (double& v : RandomNumbers) v = n01(rng);
  }
  void Solve() override {
    if (RandomNumbers.size() != (size_t)simulations_ * expansionOrder_) Initialize();
    const int R = simulations_;
    Solutions.assign((size_t)R * model_.n_dofs, 0.0);
    TipValues.assign(R, 0.0);
    Iterations.assign(R, 0);
    Residuals.assign(R, 0.0);
    const int st = MSG_MC_SOLVE_BATCH(mesh_.Handle(), model_.Poisson, kl_.Kl(), R, RandomNumbers.data(),
                                      model_.subdomain.Forces.data(),
                                      Mixed ? MSG_MODE_MIXED_BATCHED : MSG_MODE_FP64_BSR, MaxIterations, Tolerance,
                                      TipDof, Solutions.data(), TipValues.data(), Iterations.data(), Residuals.data());
    Check(st, ctx_.Handle(), "MSG_MC_SOLVE_BATCH");
  }
  std::vector<double> RandomNumbers;  // [simulations][expansionOrder]
  std::vector<double> Solutions, TipValues, Residuals;
  std::vector<int> Iterations;
  int TipDof = 0;

 private:
  friend class RaggedMonteCarloBatch;
  Context& ctx_;
  Model& model_;
  LognormalStochasticCoefficientsProvider& kl_;
  GpuMesh mesh_;
  int expansionOrder_, simulations_;

 public:
  bool Mixed;
  double Tolerance;
  int MaxIterations;

 private:
  uint64_t seed_;
};

// Several Monte Carlo analyses (models of any size or shape) in one
// MSG_MC_SOLVE_RAGGED call: each added analyzer's RandomNumbers are solved in
// the batched mixed mode to the batch's tolerance, and its Solutions,
// TipValues, Iterations and Residuals are filled as by its own Solve() on the
// same loop (the same bits alone and in the batch; a system without lattice
// numbering batched with systems that have one runs the V-cycle batch's
// standard PCG with the diagonal, the same solution to rounding). No reference
// counterpart: the reference runs one analysis, one realization after another.
class RaggedMonteCarloBatch {
 public:
  explicit RaggedMonteCarloBatch(Context& ctx, double tolerance = 1e-8, int max_iterations = 20000)
      : ctx_(ctx), Tolerance(tolerance), MaxIterations(max_iterations) {}
  void Add(MonteCarloAnalyzerWithStochasticMaterial& analyzer) { items_.push_back(&analyzer); }
  void Solve() {
    std::vector<MSG_RAGGED_SYSTEM> sys(items_.size());
    for (size_t i = 0; i < items_.size(); ++i) {
      MonteCarloAnalyzerWithStochasticMaterial& a = *items_[i];
      if (a.RandomNumbers.size() != (size_t)a.simulations_ * a.expansionOrder_) a.Initialize();
      const int R = a.simulations_;
      a.Solutions.assign((size_t)R * a.model_.n_dofs, 0.0);
      a.TipValues.assign(R, 0.0);
      a.Iterations.assign(R, 0);
      a.Residuals.assign(R, 0.0);
      MSG_RAGGED_SYSTEM& y = sys[i];
      y.mesh = a.mesh_.Handle();
      y.nu = a.model_.Poisson;
      y.kl = a.kl_.Kl();
      y.R = R;
      y.xi = a.RandomNumbers.data();
      y.b = a.model_.subdomain.Forces.data();
      y.tip_dof = a.TipDof;
      y.X = a.Solutions.data();
      y.tip = a.TipValues.data();
      y.iterations = a.Iterations.data();
      y.rel_res = a.Residuals.data();
    }
    const int st = MSG_MC_SOLVE_RAGGED(ctx_.Handle(), (int)sys.size(), sys.data(), MaxIterations, Tolerance);
    Check(st, ctx_.Handle(), "MSG_MC_SOLVE_RAGGED");
  }

 private:
  Context& ctx_;
  std::vector<MonteCarloAnalyzerWithStochasticMaterial*> items_;

 public:
  double Tolerance;
  int MaxIterations;
};

// MassAccelerationSinusoidalLoad: magnitude sin(2 pi / period * dt * i) for i
// < int(timeLength / dt), in DOF type `dof`.
struct MassAccelerationSinusoidalLoad {
  double Period, TimeStep, TimeLength, Magnitude;
  DOFType Dof;
};

// Newmark integration of every realization of a stochastic-material batch
// (the reference's coefficients and guards; the loop runs int(totalTime /
// timeStep) steps).
class NewmarkDynamicAnalyzer : public IAnalyzer {
 public:
  NewmarkDynamicAnalyzer(Context& ctx, Model& model, LognormalStochasticCoefficientsProvider& provider, double alpha,
                         double delta, double time_step, double total_time, MassAccelerationSinusoidalLoad load,
                         int simulations, double density = 1.0, double rayleigh_alpha = 0.0,
                         double rayleigh_beta = 0.0, double tolerance = 1e-8, int max_iterations = 20000)
      : ctx_(ctx), model_(model), kl_(provider), mesh_(ctx, model), simulations_(simulations), Tolerance(tolerance),
        MaxIterations(max_iterations) {
    nm_ = MSG_NEWMARK{};
    nm_.rho = density;
    nm_.rayleigh_alpha = rayleigh_alpha;
    nm_.rayleigh_beta = rayleigh_beta;
    nm_.alpha = alpha;
    nm_.delta = delta;
    nm_.dt = time_step;
    nm_.n_steps = (int)(total_time / time_step);
    nm_.acc_amp = load.Magnitude;
    nm_.acc_period = load.Period;
    nm_.acc_dof = (int)load.Dof;
    TipDof = Hexa8MeshGenerator::TipDof(model);
  }
  // InitializeCoefficients (NewmarkDynamicAnalyzer.cs:52-57): the reference's guards
  void BuildMatrices() override {
    if (nm_.delta < 0.5)
      throw InvalidOperationException(MSG_ERR_INVALID_ARGUMENT, "Newmark delta has to be bigger than 0.5.");
    const double a_limit = 0.25 * (0.5 + nm_.delta) * (0.5 + nm_.delta);
    if (nm_.alpha < a_limit)
      throw InvalidOperationException(MSG_ERR_INVALID_ARGUMENT,
                                      "Newmark alpha has to be bigger than " + std::to_string(a_limit) + ".");
  }
  void Initialize() override {
    std::mt19937_64 rng(12345);
    std::normal_distribution<double> n01(0.0, 1.0);
    RandomNumbers.resize((size_t)simulations_ * kl_.Terms());
    for (double& v : RandomNumbers) v = n01(rng);
  }
  void Solve() override {
    BuildMatrices();
    if (RandomNumbers.size() != (size_t)simulations_ * kl_.Terms()) Initialize();
    const int R = simulations_;
    TipHistory.assign((size_t)R * nm_.n_steps, 0.0);
    Solutions.assign((size_t)R * model_.n_dofs, 0.0);
    Iterations.assign(R, 0);
    const int st = MSG_NEWMARK_BATCH(mesh_.Handle(), model_.Poisson, kl_.Kl(), R, RandomNumbers.data(), &nm_, nullptr,
                                     MaxIterations, Tolerance, TipDof, TipHistory.data(), Solutions.data(),
                                     Iterations.data());
    Check(st, ctx_.Handle(), "MSG_NEWMARK_BATCH");
  }
  int Steps() const { return nm_.n_steps; }
  std::vector<double> RandomNumbers, TipHistory, Solutions;
  std::vector<int> Iterations;
  int TipDof = 0;

 private:
  Context& ctx_;
  Model& model_;
  LognormalStochasticCoefficientsProvider& kl_;
  GpuMesh mesh_;
  int simulations_;
  MSG_NEWMARK nm_;

 public:
  double Tolerance;
  int MaxIterations;
};

// The re-orthogonalising search-vector calculator
// (SolverPCGReorthogonalizationSearchVectorCalculator.cs:11-65) as a device
// store of (p, K p) pairs for one mesh, at most `capacity` pairs.
class SolverPCGReorthogonalizationSearchVectorCalculator {
 public:
  SolverPCGReorthogonalizationSearchVectorCalculator(GpuMesh& mesh, int capacity) : mesh_(mesh) {
    Check(MSG_SVS_CREATE(mesh.Handle(), capacity, &h_), mesh.Ctx().Handle(), "MSG_SVS_CREATE");
  }
  ~SolverPCGReorthogonalizationSearchVectorCalculator() {
    if (h_) MSG_SVS_DESTROY(h_);
  }
  SolverPCGReorthogonalizationSearchVectorCalculator(const SolverPCGReorthogonalizationSearchVectorCalculator&) =
      delete;
  SolverPCGReorthogonalizationSearchVectorCalculator& operator=(
      const SolverPCGReorthogonalizationSearchVectorCalculator&) = delete;
  MSG_SVS Handle() const { return h_; }
  int Count() const {
    int c = 0;
    Check(MSG_SVS_COUNT(h_, &c), mesh_.Ctx().Handle(), "MSG_SVS_COUNT");
    return c;
  }
  void ClearSearchVectors(int vectors_to_keep_from_top = 0) {
    Check(MSG_SVS_CLEAR(h_, vectors_to_keep_from_top), mesh_.Ctx().Handle(), "MSG_SVS_CLEAR");
  }

 private:
  GpuMesh& mesh_;
  MSG_SVS h_ = nullptr;
};

// SolverPCG with the re-orthogonalising calculator. StartFromStore: 0 x0 = 0;
// 1 the starting vector from the stored directions
// (InitializeStartingVectorFromSearchVectors), the store kept; 2 the same
// starting vector, then a fresh store (for a changed matrix).
class SolverPCGReorthogonalized : public SolverPCG {
 public:
  SolverPCGReorthogonalized(Context& ctx, Model& model, SolverPCGReorthogonalizationSearchVectorCalculator& search,
                            int max_iterations = 20000, double tolerance = 1e-7, int start_from_store = 0)
      : SolverPCG(ctx, model, max_iterations, tolerance), Search(search), StartFromStore(start_from_store) {}
  void Solve() override {
    Subdomain& s = model_.subdomain;
    s.Solution.assign(model_.n_dofs, 0.0);
    int it = 0;
    double rr = 0.0;
    const int st = MSG_PCG_SOLVE_REORTH(Matrix->Handle(), Search.Handle(), s.Forces.data(), s.Solution.data(),
                                        StartFromStore, MaxIterations, Tolerance, &it, &rr);
    Iterations = it;
    RelativeResidual = rr;
    Check(st, ctx_.Handle(), "MSG_PCG_SOLVE_REORTH");
  }
  SolverPCGReorthogonalizationSearchVectorCalculator& Search;
  int StartFromStore;
};

// Hexa8.CalculateStresses / CalculateForces for a batch of n elements:
// xyz [n][8][3], E [n], u (and the increment du, u when empty) [n][24] ->
// strains, stresses [n][8][6] at the Gauss points, forces [n][24].
inline void H8StressBatch(Context& ctx, const std::vector<double>& xyz, const std::vector<double>& E, double nu,
                          const std::vector<double>& u, const std::vector<double>& du, std::vector<double>& strains,
                          std::vector<double>& stresses, std::vector<double>& forces) {
  const int n = (int)E.size();
  strains.assign((size_t)n * 48, 0.0);
  stresses.assign((size_t)n * 48, 0.0);
  forces.assign((size_t)n * 24, 0.0);
  Check(MSG_H8_STRESS_BATCH(ctx.Handle(), n, xyz.data(), E.data(), nu, u.data(), du.empty() ? nullptr : du.data(),
                            strains.data(), stresses.data(), forces.data()),
        ctx.Handle(), "MSG_H8_STRESS_BATCH");
}

// PolynomialChaosSolverPCGMatrixCalculator.MultiplyWithMatrix: the stochastic
// Galerkin product over a Gaussian field's chaos basis of m variables and
// degree p, u and y block vectors [PsiSize][n_dofs].
class PolynomialChaosSolverPCGMatrixCalculator {
 public:
  PolynomialChaosSolverPCGMatrixCalculator(GpuMesh& mesh, LognormalStochasticCoefficientsProvider& provider, int m,
                                           int p)
      : mesh_(mesh), kl_(provider), m_(m), p_(p) {
    if (!provider.Gaussian())
      throw ArgumentException(MSG_ERR_INVALID_ARGUMENT,
                              "the Galerkin operator needs a GaussianStochasticCoefficientsProvider");
    Check(MSG_PC_SIZE(m, p, &psi_), nullptr, "MSG_PC_SIZE");
  }
  int PsiSize() const { return psi_; }
  std::vector<double> MultiplyWithMatrix(const std::vector<double>& u) const {
    std::vector<double> y(u.size(), 0.0);
    Check(MSG_PC_GALERKIN_MATVEC(mesh_.Handle(), mesh_.GetModel().Poisson, kl_.Kl(), m_, p_, u.data(), y.data()),
          mesh_.Ctx().Handle(), "MSG_PC_GALERKIN_MATVEC");
    return y;
  }

 private:
  GpuMesh& mesh_;
  LognormalStochasticCoefficientsProvider& kl_;
  int m_, p_, psi_ = 0;
};

// Continuous-batching service of independent realizations (MSG_SERVE_*; no
// counterpart in the reference, whose realization loop is sequential). Models
// are registered once; each request is one realization (its xi row), queued,
// run in a free slot of its model's batch and polled for its displacements.
class Server {
 public:
  struct Result {
    int Status = MSG_PENDING;
    std::vector<double> X;
    int Iterations = 0;
    double RelativeResidual = 0.0, LatencyMs = 0.0;
  };
  Server(Context& ctx, int max_batch = 64) : ctx_(ctx) {
    Check(MSG_SERVE_START(ctx.Handle(), max_batch), ctx.Handle(), "MSG_SERVE_START");
  }
  ~Server() { MSG_SERVE_STOP(ctx_.Handle()); }
  Server(const Server&) = delete;
  Server& operator=(const Server&) = delete;
  // the model's mesh stays alive with the server
  int AddModel(Model& model, LognormalStochasticCoefficientsProvider& provider, double tolerance = 1e-8,
               int max_iterations = 20000) {
    meshes_.emplace_back(new GpuMesh(ctx_, model));
    int id = -1;
    Check(MSG_SERVE_ADD_MODEL(ctx_.Handle(), meshes_.back()->Handle(), model.Poisson, provider.Kl(),
                              model.subdomain.Forces.data(), tolerance, max_iterations, &id),
          ctx_.Handle(), "MSG_SERVE_ADD_MODEL");
    dofs_.push_back(model.n_dofs);
    return id;
  }
  MSG_REQ Submit(int model_id, const std::vector<double>& xi) {
    MSG_REQ id = 0;
    Check(MSG_SERVE_SUBMIT(ctx_.Handle(), model_id, xi.data(), &id), ctx_.Handle(), "MSG_SERVE_SUBMIT");
    requests_.push_back({id, model_id});
    return id;
  }
  // lanes of a model (-1: all) admitting requests; lanes added and retired so far
  struct Lanes {
    int Active = 0;
    int64_t Added = 0, Retired = 0;
  };
  Lanes LaneCount(int model_id = -1) {
    Lanes l;
    Check(MSG_SERVE_LANES(ctx_.Handle(), model_id, &l.Active, &l.Added, &l.Retired), ctx_.Handle(),
          "MSG_SERVE_LANES");
    return l;
  }
  // timeout_ms < 0 waits until the request is done; a finished request that
  // did not converge or was cancelled throws as the other calls do
  Result Poll(MSG_REQ id, int timeout_ms = -1) {
    Result r;
    r.X.assign(dofs_.at(ModelOf(id)), 0.0);
    r.Status = MSG_SERVE_POLL(ctx_.Handle(), id, timeout_ms, r.X.data(), &r.Iterations, &r.RelativeResidual,
                              &r.LatencyMs);
    if (r.Status != MSG_PENDING) Check(r.Status, ctx_.Handle(), "MSG_SERVE_POLL");
    return r;
  }
  void Cancel(MSG_REQ id) { Check(MSG_SERVE_CANCEL(ctx_.Handle(), id), ctx_.Handle(), "MSG_SERVE_CANCEL"); }

 private:
  int ModelOf(MSG_REQ id) const {
    for (const auto& q : requests_)
      if (q.first == id) return q.second;
    throw ArgumentException(MSG_ERR_INVALID_ARGUMENT, "unknown request");
  }
  Context& ctx_;
  std::vector<std::unique_ptr<GpuMesh>> meshes_;
  std::vector<int> dofs_;
  std::vector<std::pair<MSG_REQ, int>> requests_;
};

}  // namespace msolve
