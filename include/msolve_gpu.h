/*
 * msolve_gpu.h -- C ABI of the B200 (sm_100a) Hexa8 linear-elastic solve path.
 *
 * The drop-in boundary for MSolve's Hexa8 static solve and its Monte Carlo
 * realization loop. Every entry point is extern "C", Cdecl, takes plain
 * pointers and sizes, and returns an int status (0 = ok; negative codes below,
 * message through MSG_LAST_ERROR). It is written to be bound from C# with
 * [DllImport("msolve_gpu", CallingConvention = CallingConvention.Cdecl)], the
 * convention the reference already uses for its native element library
 * (ISAAR.MSolve.PreProcessor/Elements/Hexa8.cs:26-62).
 *
 * Conventions
 *  - Host pointers unless an entry point says "device". Host buffers are
 *    caller-owned and only read/written during the call.
 *  - Element node order and packed 24x24 layout are the reference's:
 *    nodes (-,-,-),(+,-,-),(+,+,-),(-,+,-),(-,-,+),(+,-,+),(+,+,+),(-,+,+)
 *    (FEMElements/FEMElements/rElHexa8.f90:43-68), element DOFs node-major x,y,z,
 *    packed row-wise upper triangle of 300 entries
 *    (ISAAR.MSolve.Matrices/SymmetricMatrix2D.cs:22-49).
 *  - DOF numbering is the caller's (Model/Subdomain numbering, constrained = -1,
 *    ISAAR.MSolve.PreProcessor/Subdomain.cs:77-135). Vectors of length n_dofs are
 *    in that numbering.
 *  - Handles are bound to the context (one CUDA device, one stream). Calls on
 *    one context are serialised by an internal mutex; different contexts may be
 *    used from different threads.
 */
#ifndef MSOLVE_GPU_H
#define MSOLVE_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes. The first three reuse FEMElements/FEMElements/hCommon.h:18-29. */
#define MSG_OK                    0
#define MSG_ERR_UNKNOWN          (-1)     /* iErrUnknown */
#define MSG_ERR_OUT_OF_MEMORY    (-100)   /* iErrNotEnoughMemory (device or memory budget) */
#define MSG_ERR_NEG_DET          (-1001)  /* iErrNegDet: Jacobian determinant < 1e-8 */
#define MSG_ERR_NOT_CONVERGED    (-2001)  /* PCG hit max iterations above tolerance */
#define MSG_ERR_BREAKDOWN        (-2002)  /* p.q <= 0 or NaN in PCG */
#define MSG_ERR_TIMEOUT          (-2003)  /* a bounded device/host wait gave up */
#define MSG_ERR_CANCELLED        (-2004)  /* serving request cancelled */
#define MSG_ERR_INVALID_ARGUMENT (-2005)
#define MSG_ERR_CUDA             (-2006)  /* CUDA runtime error (message has the text) */
#define MSG_ERR_NOT_STRUCTURED   (-2007)  /* batched matrix-free path needs a structured cube lattice */
#define MSG_ERR_NO_DEVICE        (-2008)

/* ---- solver modes for MSG_MC_SOLVE_BATCH */
#define MSG_MODE_FP64_BSR        0  /* plain FP64: per realization assemble BSR + Jacobi-PCG (the drop-in) */
#define MSG_MODE_MIXED_BATCHED   1  /* all realizations at once: matrix-free FP32 PCG + FP64 refinement */

typedef struct msg_context* MSG_CTX;
typedef struct msg_mesh* MSG_MESH;
typedef struct msg_matrix* MSG_MAT;
typedef struct msg_svs* MSG_SVS;

/* ------------------------------------------------------------------ context */
/* Create a context on CUDA device `device`. mem_budget_bytes = 0 means no budget
 * beyond the device's free memory. The batched entry points keep their device
 * buffers in the context from one call to the next (grown to the largest call,
 * never shrunk; charged to the budget) so that repeated calls allocate
 * nothing; they are released with the context (MSG_DESTROY). No counterpart
 * in the reference (which has no device); the C# shim creates one per solver
 * instance. */
int MSG_CREATE(int device, uint64_t mem_budget_bytes, MSG_CTX* out);
int MSG_DESTROY(MSG_CTX ctx);
/* Text of the last error on this context (valid until the next call on it). */
const char* MSG_LAST_ERROR(MSG_CTX ctx);
/* ABI version (major*10000 + minor*100 + patch). */
int MSG_VERSION(void);

/* ------------------------------------------------------------------ element kernels */
/* Batched twin of CALCH8GAUSSMATRICES + CALCH8K
 * (FEMElements/FEMElements/rElHexa8.f90:422-464, 489-543; called from
 * Hexa8WithStochasticMaterial.StiffnessMatrix, Hexa8WithStochasticMaterial.cs:61-110):
 * for each of n elements, isotropic D(E[e], nu) at every 2x2x2 Gauss point,
 * K_e = sum_gp w B^T D B, packed 300 entries.
 * xyz [n][8][3], E [n], Ke [n][300]. Returns MSG_ERR_NEG_DET if any element has
 * detJ < 1e-8 at a Gauss point (Ke is still written, as the Fortran does). */
int MSG_H8_KE_BATCH(MSG_CTX ctx, int n, const double* xyz, const double* E, double nu, double* Ke);

/* Batched consistent mass, Hexa8.CalculateConsistentMass
 * (ISAAR.MSolve.PreProcessor/Elements/Hexa8.cs:403-435): xyz [n][8][3], Me [n][300]. */
int MSG_H8_ME_BATCH(MSG_CTX ctx, int n, const double* xyz, double rho, double* Me);

/* Batched stress recovery, Hexa8.CalculateStresses + Hexa8.CalculateForces
 * (ISAAR.MSolve.PreProcessor/Elements/Hexa8.cs:453-510) over CALCH8STRAINS and
 * CALCH8FORCES (FEMElements/FEMElements/rElHexa8.f90:636-648, 724-747) with the
 * elastic material (ElasticMaterial3D.cs:20-44, 75-81): per element and 2x2x2
 * Gauss point (xi outer, zeta inner) strains = B u (exx, eyy, ezz, gxy, gyz,
 * gzx), stresses = D(E, nu) B du (the material stores the strain increment),
 * and internal forces = sum_gp w B^T stresses (24). xyz [n][8][3], E [n],
 * u [n][24], du [n][24] (NULL: du = u). Outputs (each may be NULL): strains,
 * stresses [n][8][6], forces [n][24]. MSG_ERR_NEG_DET as MSG_H8_KE_BATCH. */
int MSG_H8_STRESS_BATCH(MSG_CTX ctx, int n, const double* xyz, const double* E, double nu, const double* u,
                        const double* du, double* strains, double* stresses, double* forces);
/* The same for every element of the mesh and every realization of a batch, on
 * the device: E_dev [R][n_elems] (MSG_KL_FIELD layout), X_dev [R][n_dofs] (the
 * solutions of MSG_MC_SOLVE_BATCH_DEVICE; constrained DOFs are 0), du = u.
 * Outputs (device, each may be NULL): strains_dev, stresses_dev
 * [R][n_elems][8][6], forces_dev [R][n_elems][24]. The reference's stochastic
 * material reports zero stresses (StochasticElasticMaterial3D.cs:75); this
 * returns the elastic stresses of each realization's field. */
int MSG_STRESS_BATCH_DEVICE(MSG_MESH mesh, int R, const double* E_dev, double nu, const double* X_dev,
                            double* strains_dev, double* stresses_dev, double* forces_dev);

/* ------------------------------------------------------------------ mesh */
/* Upload a Hexa8 mesh: xyz [n_nodes][3], conn [n_elems][8] (0-based node
 * indices), dof [n_nodes][3] (free DOF number or -1 if constrained, the
 * Subdomain.NodalDOFsDictionary numbering). Builds the 3x3-block sparsity
 * pattern (replacing GlobalMatrixAssemblerSkyline.CalculateRowIndex,
 * GlobalMatrixAssemblerSkyline.cs:14-42) and detects whether the mesh is a
 * structured lattice of equal cubes in generator order
 * (Hexa8MeshGenerator.BuildNodes / element loop, Hexa8MeshGenerator.cs:508-568,
 * 1075-1089), which enables MSG_MODE_MIXED_BATCHED. */
int MSG_MESH_CREATE(MSG_CTX ctx, int n_nodes, const double* xyz, int n_elems, const int* conn,
                    const int* dof, int n_dofs, MSG_MESH* out);
/* info[0]=structured(0/1) info[1..3]=nx,ny,nz info[4]=n_dofs info[5]=n_block_rows
 * info[6]=nnz_blocks info[7]=n_elems. (8 ints) */
int MSG_MESH_INFO(MSG_MESH mesh, int64_t* info8);
int MSG_MESH_DESTROY(MSG_MESH mesh);

/* ------------------------------------------------------------------ assembled FP64 operator */
/* Assemble the global stiffness in 3x3 block sparse form on the device from
 * per-element Young's moduli E [n_elems] and nu: element matrices by the
 * MSG_H8_KE_BATCH kernel, summed per block in a fixed order (deterministic).
 * Replaces ProblemStructural.BuildKs -> GlobalMatrixAssemblerSkyline.CalculateGlobalMatrix
 * (ProblemStructural.cs:63-89; GlobalMatrixAssemblerSkyline.cs:51-103). */
int MSG_ASSEMBLE_BSR(MSG_MESH mesh, const double* E, double nu, MSG_MAT* out);
/* Same, from caller-supplied element matrices Ke [n_elems][300] (host), the
 * IElementMatrixProvider seam (ISAAR.MSolve.PreProcessor/Interfaces/IElementMatrixProvider.cs:9-12). */
int MSG_ASSEMBLE_BSR_KE(MSG_MESH mesh, const double* Ke, MSG_MAT* out);
/* y = K x in DOF numbering (IMatrix2D.Multiply parity, SkylineMatrix2D.cs:224-286). */
int MSG_MAT_MULTIPLY(MSG_MAT mat, const double* x, double* y);
/* diag [n_dofs] = K_jj (the Jacobi preconditioner's source,
 * PolynomialChaosSolverPCGMatrixCalculator.cs:467-495). */
int MSG_MAT_DIAGONAL(MSG_MAT mat, double* diag);
int MSG_MAT_DESTROY(MSG_MAT mat);

/* Jacobi-preconditioned PCG with the reference's semantics
 * (ISAAR.MSolve.Solvers/PCG/SolverPCG.cs:105-149, simple search vector
 * SolverPCGSimpleSearchVectorCalculator.cs:18-41): x0 = 0, r0 = b, stop when
 * ||r_k|| / ||b|| < tol on the recursively updated r, skip if ||b|| <= 1e-25.
 * The whole loop runs on the device: one CUDA graph launch a solve, whose
 * conditional WHILE node repeats 8-iteration rounds until the solve ends (no
 * host round trip between iterations or rounds).
 * iterations = the reference's count (loop index at the break); rel_res = last
 * ||r||/||b||. Returns MSG_ERR_NOT_CONVERGED if max_it was reached. */
int MSG_PCG_SOLVE(MSG_MAT mat, const double* b, double* x, int max_it, double tol, int* iterations,
                  double* rel_res);

/* MSG_PCG_SOLVE with the matrix values and the loop's vectors in FP32 (half
 * the bytes of the dominant SpMV traffic) and FP64 refinement: the iterate x is
 * FP64, accumulated from an FP32 correction, and every dot product is summed in
 * FP64; two kernels an iteration (the FP32 SpMV with alpha and beta from its
 * partials, then one update pass that also forms the next direction). When the
 * recursive residual has dropped by "reliable_delta" (or below tol) it is
 * replaced by the FP64 true residual b - K x computed with the FP64 values,
 * the search direction is kept, and the solve stops only when
 * ||b - K x|| / ||b|| < tol in FP64 (rel_res). iterations counts as
 * MSG_PCG_SOLVE. The FP32 copy of the values is built on first use. Like
 * MSG_PCG_SOLVE, one CUDA graph launch a solve; the true-residual step is a
 * conditional node of that graph. No counterpart in the reference. */
int MSG_PCG_SOLVE_MIXED(MSG_MAT mat, const double* b, double* x, int max_it, double tol, int* iterations,
                        double* rel_res);

/* Search vectors kept across solves: SolverPCGReorthogonalizationSearchVectorCalculator
 * (ISAAR.MSolve.Solvers/PCG/SolverPCGReorthogonalizationSearchVectorCalculator.cs:11-65)
 * holds every direction p and K p of the solves it served; here a device store of at
 * most `capacity` pairs for one mesh. MSG_SVS_CLEAR keeps the `keep_from_top` oldest
 * pairs (ClearSearchVectors, :36-63; < 1 clears all). */
int MSG_SVS_CREATE(MSG_MESH mesh, int capacity, MSG_SVS* out);
int MSG_SVS_CLEAR(MSG_SVS store, int keep_from_top);
int MSG_SVS_COUNT(MSG_SVS store, int* count);
int MSG_SVS_DESTROY(MSG_SVS store);
/* SolverPCG (ISAAR.MSolve.Solvers/PCG/SolverPCG.cs:105-149) with the
 * re-orthogonalising search-vector calculator (SearchVectors.cs:13-166): each new
 * direction is z - sum_c (z.q_c / p_c.q_c) p_c over every stored pair, the gradient
 * is (p.r)/(p.q) and each (p, q) is appended to the store; Jacobi preconditioner,
 * FP64, stop on the recursive ||r||/||b|| < tol, iteration count = loop index at
 * the break (as MSG_PCG_SOLVE). start_from_store = 1:
 * InitializeStartingVectorFromReorthogonalizedSearchVectors (:115-166; drops the
 * last pair, x0 = sum_c (p_c.b / p_c.q_c) p_c), then r0 = b - K x0.
 * start_from_store = 2: the same starting vector, then the store is emptied: the
 * pairs are K-conjugate only for the matrix that produced them, so a changed
 * matrix (the next Monte Carlo realization) takes them as an initial guess but
 * must not re-orthogonalise against them. b, x [n_dofs] (host).
 * MSG_ERR_OUT_OF_MEMORY when the store fills up during the solve. */
int MSG_PCG_SOLVE_REORTH(MSG_MAT mat, MSG_SVS store, const double* b, double* x, int start_from_store, int max_it,
                         double tol, int* iterations, double* rel_res);

/* MSG_PCG_SOLVE without device allocation. No counterpart in the reference.
 * For callers that must not allocate device memory while solving: cudaMalloc
 * and cudaFree synchronise the whole device (a caller overlapping other GPU
 * work would stall), and a host that hands the library a fixed share of device
 * memory may forbid allocations outside it. b_dev and x_dev are the caller's
 * device buffers (n_dofs doubles, DOF numbering); the solve's working vectors
 * live in one fixed device array of the library (about 9.5 MB, held on every
 * GPU that loads the library until the process exits), which limits the mesh
 * to 65536 nodes (larger meshes: MSG_ERR_INVALID_ARGUMENT). MSG_CREATE looks up
 * that array's device address, so the solve itself does no set-up. Stream
 * ordering: the call runs on the context's own stream, which does not wait for
 * other streams (not even the legacy default stream), so the caller's writes
 * to b_dev must be complete before the call (synchronise the stream that wrote
 * it) and x_dev must not be in use by other GPU work; the call returns after
 * its stream has finished, so x_dev holds the solution on return. All calls
 * share the array, which keeps the previous call's contents (the call clears
 * what must start at zero): calls whose GPU work overlaps (two host threads on
 * two contexts of the same device) race and must be serialised by the caller.
 * Semantics, kernels and results as MSG_PCG_SOLVE, including the
 * MSG_ERR_NOT_CONVERGED / MSG_ERR_BREAKDOWN returns with x_dev, iterations and
 * rel_res written. */
int MSG_PCG_SOLVE_NOALLOC(MSG_MAT mat, const double* b_dev, double* x_dev, int max_it, double tol, int* iterations,
                          double* rel_res);

/* ------------------------------------------------------------------ stochastic field */
/* Separable Karhunen-Loeve table of a lognormal Young's modulus, the content of
 * the eigen-data file read by LognormalFileStochasticCoefficientsProvider
 * (ISAAR.MSolve.PreProcessor/Stochastic/LognormalFileStochasticCoefficientsProvider.cs:71-118):
 * per term k and axis a: frequency w3[k][a], amplitude amp3[k][a], 1-based 1-D
 * mode index idx3[k][a] (odd -> cos, even -> sin), eigenvalue eig[k].
 * E(x) = exp(ln(mean) - mc*sigma^2/2 + sum_k xi_k sigma sqrt(eig_k)
 *            prod_a amp * {cos|sin}(w * (x_a - domain_a/2)))   (GetCoefficient :173-193)
 * evaluated at each element's bounding-box centre (Hexa8WithStochasticMaterial.cs:112-140). */
typedef struct {
  int n_terms;          /* 1..64 */
  const double* w3;
  const double* amp3;
  const int* idx3;
  const double* eig;
  double domain[3];
  double mean;
  double sigma;
  int mean_correction; /* 1: reference form ln(mean) - sigma^2/2; 0: exp(sigma g) */
  /* 0: lognormal field (LognormalFileStochasticCoefficientsProvider); 1: Gaussian
   * field E = mean (1 + sum_k xi_k sigma sqrt(eig_k) phi_k(x)), the coefficient of
   * GaussianFileStochasticCoefficientsProvider.GetCoefficient
   * (ISAAR.MSolve.PreProcessor/Stochastic/GaussianFileStochasticCoefficientsProvider.cs:72-108,
   * sigma = its covariance 0.15), so K(E) = K_0 + sum_k xi_k K_k is the matrix
   * MonteCarloAnalyzer composes (ISAAR.MSolve.Analyzers/MonteCarloAnalyzer.cs:88-172);
   * mean_correction is ignored. E must stay positive for the solvers. */
  int gaussian;
} MSG_KL;

/* Build the KL table of the separable exponential kernel exp(-sum|dx_a|/corr_len)
 * on [0,domain] (analytic 1-D eigen-pairs, n1d modes per axis, the n_terms
 * largest 3-D products). Outputs into the caller's arrays w3/amp3/idx3 [n_terms][3], eig [n_terms]. */
int MSG_KL_TABLE(const double* domain3, double corr_len, int n_terms, int n1d, double* w3, double* amp3,
                 int* idx3, double* eig);
/* E [R][n_elems] for xi [R][n_terms] (the MC loop's RandomVariables,
 * MonteCarloAnalyzerWithStochasticMaterial.cs:258-261). */
int MSG_KL_FIELD(MSG_MESH mesh, const MSG_KL* kl, int R, const double* xi, double* E);

/* ------------------------------------------------------------------ polynomial chaos (Gaussian) */
/* Basis of PolynomialChaosCoefficientsCalculator (ISAAR.MSolve.PreProcessor/Stochastic/
 * PolynomialChaosCoefficientsCalculator.cs:30-300): the multi-indices of m Gaussian
 * variables up to total degree p in the reference's order (P = MSG_PC_SIZE of them,
 * basis [P][m]) and their squared norms prod_l alpha_l! (norms [P]). */
int MSG_PC_SIZE(int m, int p, int* size);
int MSG_PC_BASIS(int m, int p, int* basis, int* norms);
/* The stochastic Galerkin product y = A u of PolynomialChaosSolverPCGMatrixCalculator.
 * MultiplyWithMatrix (ISAAR.MSolve.Analyzers/PolynomialChaosSolverPCGMatrixCalculator.cs:1062-1089,
 * Gaussian branch): y_j = <psi_j^2> K_0 u_j + sum_i sum_k <xi_i psi_j psi_k> K_i u_k,
 * with K_0 the stiffness of the mean modulus and K_i that of the i-th KL term
 * (kl->gaussian = 1, the first m terms; the Monte Carlo composition's matrices),
 * applied element by element on a structured lattice in FP64. u, y: block-major
 * [P][n_dofs] (host), the reference's vector layout. */
int MSG_PC_GALERKIN_MATVEC(MSG_MESH mesh, double nu, const MSG_KL* kl, int m, int p, const double* u, double* y);

/* ------------------------------------------------------------------ Monte Carlo batch */
/* The realization loop of MonteCarloAnalyzerWithStochasticMaterial.SolveNormal
 * (ISAAR.MSolve.Analyzers/MonteCarloAnalyzerWithStochasticMaterial.cs:232-296):
 * for each realization r: E field from xi[r], rebuild K, solve K x_r = b.
 *   mode MSG_MODE_FP64_BSR: realizations one after another, FP64 BSR + Jacobi PCG
 *     (recursive-residual stop as MSG_PCG_SOLVE).
 *   mode MSG_MODE_MIXED_BATCHED: all realizations in one batch on a structured
 *     cube lattice: matrix-free FP32 element-by-element operator inside PCG
 *     (per-realization geometric multigrid V-cycle preconditioner by default,
 *     Jacobi with MSG_SET_OPTION "multigrid" = 0), FP64 true residual
 *     r = b - K x and FP64 solution update (iterative refinement); stop when
 *     ||b - K x||/||b|| < tol in FP64. On a mesh that is not a cube lattice
 *     (distorted or unstructured Hexa8) all realizations are solved at once
 *     by PCG over an element-by-element operator (each element's stiffness
 *     at E = 1 computed once, scaled by E per realization; FP32 loop, FP64
 *     iterate and true residuals) to the same FP64 stopping rule; the
 *     preconditioner is the multigrid V-cycle of the cube lattice with the
 *     same numbering when the mesh has the generator's numbering and element
 *     order (nodes moved) and that lattice coarsens (MSG_SET_OPTION
 *     "multigrid" != 0), Jacobi otherwise;
 *     with MSG_SET_OPTION "element_batch" = 0 one after another with the
 *     assembled FP32-value PCG and FP64 refinement of MSG_PCG_SOLVE_MIXED.
 * xi [R][kl->n_terms], b [n_dofs]. Outputs (each may be NULL): X [R][n_dofs],
 * tip [R] = X[r][tip_dof], iterations [R] (matrix products per realization),
 * rel_res [R] (final FP64 ||b - K x||/||b||). A realization that does not
 * converge or breaks down (p.q <= 0 or NaN, e.g. from a NaN modulus) makes the
 * call return MSG_ERR_NOT_CONVERGED or MSG_ERR_BREAKDOWN; the outputs of the
 * other realizations are still complete. */
int MSG_MC_SOLVE_BATCH(MSG_MESH mesh, double nu, const MSG_KL* kl, int R, const double* xi, const double* b,
                       int mode, int max_it, double tol, int tip_dof, double* X, double* tip, int* iterations,
                       double* rel_res);
/* Device-pointer variant (xi_dev, b_dev, X_dev on this context's device; X_dev may
 * be NULL). Host outputs tip/iterations/rel_res as above. For callers that keep
 * inputs and results resident in device memory. */
int MSG_MC_SOLVE_BATCH_DEVICE(MSG_MESH mesh, double nu, const MSG_KL* kl, int R, const double* xi_dev,
                              const double* b_dev, int mode, int max_it, double tol, int tip_dof, double* X_dev,
                              double* tip, int* iterations, double* rel_res);

/* MSG_MC_SOLVE_BATCH with the copy of X to the host left in flight: the copy
 * runs on a copy stream of the context (from one of two device output buffers)
 * while the caller prepares and submits the next batch. tip, iterations and
 * rel_res are complete on return; X is complete when the next
 * MSG_MC_SOLVE_BATCH_PIPELINED on the context returns, or after
 * MSG_MC_FLUSH. So consecutive pipelined calls need different X buffers, and
 * X should be page-locked host memory (a pageable X makes the copy
 * synchronous). MSG_MC_SOLVE_BATCH and MSG_DESTROY flush first. No reference
 * counterpart (the reference returns each realization's solution before the
 * next starts). */
int MSG_MC_SOLVE_BATCH_PIPELINED(MSG_MESH mesh, double nu, const MSG_KL* kl, int R, const double* xi,
                                 const double* b, int mode, int max_it, double tol, int tip_dof, double* X,
                                 double* tip, int* iterations, double* rel_res);
/* Waits until the X of every pipelined call on the context is on the host. */
int MSG_MC_FLUSH(MSG_CTX ctx);

/* One system of a ragged batch: a Hexa8 mesh of any shape and size (of the
 * context the batch runs on), its material and KL field, R realizations and
 * the load. Host buffers: xi [R][kl->n_terms], b [n_dofs]; outputs (each may
 * be NULL) X [R][n_dofs], tip [R] = X[r][tip_dof], iterations [R] (operator
 * products), rel_res [R] (final FP64 ||b - K x||/||b||). */
typedef struct {
  MSG_MESH mesh;
  double nu;
  const MSG_KL* kl;
  int R;
  const double* xi;
  const double* b;
  int tip_dof;
  double* X;
  double* tip;
  int* iterations;
  double* rel_res;
} MSG_RAGGED_SYSTEM;
/* The realization loop of MonteCarloAnalyzerWithStochasticMaterial.SolveNormal
 * (ISAAR.MSolve.Analyzers/MonteCarloAnalyzerWithStochasticMaterial.cs:232-296)
 * for several systems of uneven mesh size at once. Structured cube lattices go
 * through the lattice loop of MSG_MC_SOLVE_BATCH (mixed mode, the same results
 * as that call) unless the "ragged_lattice_loop" option is 0: with the
 * "ragged_side_by_side" option on (the default) their loops are stepped side
 * by side, each on its own stream with its own buffers and loop graph (kept in
 * the context for the next call), on a second host thread while the calling
 * thread runs the other systems' batch, each lattice taking the steps it
 * takes alone (the same bits); with it off, one lattice after another and
 * then the other systems. For the other
 * systems every iteration of every realization runs in the same three persistent launches
 * (element-by-element FP32 operator over each element's stiffness at E = 1
 * scaled by E per realization, per-realization scalars, fused vector update),
 * eight iterations to a CUDA graph launch, Jacobi-preconditioned CG (the
 * reference's SolverPCG with the diagonal preconditioner) with the iterate in
 * FP64 and FP64 true residuals, to ||b - K x||/||b|| < tol in FP64 for each
 * realization. With the multigrid option on (the default), a system whose mesh
 * has the numbering of an nx x ny x nz lattice with every side even and >= 4
 * (moved nodes allowed) is preconditioned instead by the V-cycle of its cube
 * lattice, and then the whole batch runs standard PCG (the operator, scalar
 * and vector launches shared, one V-cycle per such system, the diagonal for
 * the others; two iterations to a graph launch). A system's results do not
 * depend on the other systems in the batch: the same bits alone and in any mix
 * of systems, except that a system without a V-cycle takes the fused Jacobi
 * loop when no system of its batch has one (the same solution to rounding). No
 * reference counterpart as an entry point (the reference solves one
 * realization after another). Returns MSG_ERR_NOT_CONVERGED or
 * MSG_ERR_BREAKDOWN as MSG_MC_SOLVE_BATCH, with every other output complete. */
int MSG_MC_SOLVE_RAGGED(MSG_CTX ctx, int n_systems, const MSG_RAGGED_SYSTEM* systems, int max_it, double tol);

/* ------------------------------------------------------------------ Newmark batch */
/* Parameters of NewmarkDynamicAnalyzer (ISAAR.MSolve.Analyzers/NewmarkDynamicAnalyzer.cs:38-77)
 * with the structural provider's effective matrix K + a0 M + a1 C
 * (ProblemStructural.cs:138-157), Hexa8 consistent mass and Rayleigh damping
 * C_e = rayleigh_alpha M_e + rayleigh_beta K_e (Hexa8.cs:403-451), and one
 * MassAccelerationSinusoidalLoad (MassAccelerationSinusoidalLoad.cs:17-20):
 * ground acceleration acc_amp sin(2 pi / acc_period * dt * i) in DOF acc_dof at
 * step i, applied as the inertial load sum_e M_e a_g (Hexa8.cs:512-530). */
typedef struct {
  double rho;            /* density of the consistent mass */
  double rayleigh_alpha; /* mass-proportional damping */
  double rayleigh_beta;  /* stiffness-proportional damping */
  double alpha;          /* Newmark alpha (>= (0.5 + delta)^2 / 4), 0.25: average acceleration */
  double delta;          /* Newmark delta (>= 0.5) */
  double dt;             /* time step */
  int n_steps;           /* the reference runs (int)(totalTime / dt) steps */
  double acc_amp;
  double acc_period;
  int acc_dof;           /* 0 X, 1 Y, 2 Z */
} MSG_NEWMARK;

/* Newmark integration of R realizations at once (the batched counterpart of
 * NewmarkDynamicAnalyzer.Solve, :280-315, for a stochastic material: E field
 * of realization r from xi[r] as in MSG_MC_SOLVE_BATCH). Every step solves the
 * effective system of all realizations with the mixed batched PCG to the FP64
 * true relative residual tol, started from the Newmark predictor of the new
 * displacement (option "newmark_predictor"; 0: from the previous displacement;
 * the reference restarts SolverPCG from zero; all stop on the same criterion). Structured cube lattices only (MSG_ERR_NOT_STRUCTURED otherwise).
 * xi [R][kl->n_terms]; f_static [n_dofs] static nodal loads added every step
 * (Model.AssignLoads) or NULL. Outputs (each may be NULL): tip_hist
 * [R][n_steps] displacement of DOF tip_dof after each step, U [R][n_dofs] final
 * displacements, iterations [R] operator products summed over the steps. */
int MSG_NEWMARK_BATCH(MSG_MESH mesh, double nu, const MSG_KL* kl, int R, const double* xi, const MSG_NEWMARK* nm,
                      const double* f_static, int max_it, double tol, int tip_dof, double* tip_hist, double* U,
                      int* iterations);

/* ------------------------------------------------------------------ serving */
/* Continuous-batching service on a context. No counterpart in the reference
 * (its realization loop is sequential, MonteCarloAnalyzerWithStochasticMaterial.cs:258-276).
 * A model is a structured mesh with its material (nu), KL table and load b
 * [n_dofs]; a request is one realization of a model (its xi [kl->n_terms]).
 * Requests wait in their model's queue, enter a free slot of one of the
 * model's lanes at the next chunk boundary and leave as soon as their own FP64
 * true residual is below the model's tol. A lane is a batch of max_batch slots
 * (rounded up to 64) with its device state; admission is by device memory: a
 * model's first lane is allocated when the model is added (against the
 * context's memory budget, MSG_CREATE), a manager thread adds lanes (at most 8
 * a model) while a model's queue outgrows its free slots and the budget has
 * room, and retires idle extra lanes when another model's requests need the
 * memory or after a second without work. A request's arithmetic does not
 * depend on the other requests in flight or on its lane: results are bitwise
 * identical alone or mixed. One worker thread per lane runs its batch on the
 * lane's own stream; every entry point may be called from any thread. */
#define MSG_PENDING 1 /* MSG_SERVE_POLL: not finished yet (not an error) */
typedef uint64_t MSG_REQ;
int MSG_SERVE_START(MSG_CTX ctx, int max_batch);
/* Register a model; *model_id identifies it in MSG_SERVE_SUBMIT. b is copied. */
int MSG_SERVE_ADD_MODEL(MSG_CTX ctx, MSG_MESH mesh, double nu, const MSG_KL* kl, const double* b, double tol,
                        int max_it, int* model_id);
/* Queue one realization (xi is copied); *id names the request. */
int MSG_SERVE_SUBMIT(MSG_CTX ctx, int model_id, const double* xi, MSG_REQ* id);
/* Wait up to timeout_ms (0: do not wait, < 0: until done) for request id.
 * Finished: copies X [n_dofs] (may be NULL), iterations (operator products),
 * rel_res (final FP64 ||b - K x|| / ||b||) and latency_ms (submit to finish),
 * forgets the request and returns MSG_OK, MSG_ERR_NOT_CONVERGED,
 * MSG_ERR_BREAKDOWN or MSG_ERR_CANCELLED. Not finished: MSG_PENDING. */
int MSG_SERVE_POLL(MSG_CTX ctx, MSG_REQ id, int timeout_ms, double* X, int* iterations, double* rel_res,
                   double* latency_ms);
/* Cancel a request: a queued one never runs, a running one leaves its slot at
 * the next chunk boundary; its poll returns MSG_ERR_CANCELLED. */
int MSG_SERVE_CANCEL(MSG_CTX ctx, MSG_REQ id);
/* Requests waiting in the queues and occupying slots. */
int MSG_SERVE_STATS(MSG_CTX ctx, int64_t* queued, int64_t* running);
/* Lanes of model model_id (-1: all models) that currently admit requests, and
 * the lanes added and retired since MSG_SERVE_START. No reference counterpart. */
int MSG_SERVE_LANES(MSG_CTX ctx, int model_id, int* lanes, int64_t* added, int64_t* retired);
/* Stop the worker and free every model (pending requests are dropped). */
int MSG_SERVE_STOP(MSG_CTX ctx);

/* Tunables of the mixed solver on this context: "reliable_delta" (the FP32
 * recursive residual may fall by this factor before it is replaced by the FP64
 * true residual, default 0.1), "chunk" (FP32 iterations per CUDA-graph launch,
 * even, default 16), "fixed_updates" (1: the FP64 true-residual step runs after every chunk for
 * every realization, so each realization's arithmetic no longer depends on the
 * rest of the batch: bitwise identical alone or batched; default 0: the step
 * runs when some realization asks for it), "multigrid" (preconditioner of the
 * batched lattice loop: 1, default, a geometric multigrid V-cycle for systems
 * without a mass term (static solves, serving), Jacobi for those with one
 * (Newmark); 2: the V-cycle for both; 0: Jacobi for both. The V-cycle needs a
 * lattice whose element counts are even at least once; otherwise Jacobi runs),
 * "multigrid_levels" (lattice levels at most, fine level included, 2..6,
 * default 6; a level halves every axis while each keeps at least 2 elements),
 * "multigrid_sweeps" (damped Jacobi sweeps on the coarsest level, default 20),
 * "multigrid_omega" (Jacobi damping of every level, 0 = derived from the
 * element stiffness, default), "multigrid_delta" (reliable-update factor of the
 * V-cycle-preconditioned loops, default 0.001; their inner chunk is 2 iterations), "multigrid_packed"
 * (1, default: the three level-0 operator passes of an iteration work on two
 * realizations per thread with packed FP32 arithmetic; 0: one per thread),
 * "multigrid_fused_coarse" (1, default: every sweep of the coarsest level in
 * one launch when that level has at most 3 x 3 nodes across y and z; 0: one
 * launch per sweep; the results are identical), "serve_persistent" (serving
 * lanes created afterwards: 1, default, persistent grids of one CTA per SM;
 * 0: one CTA per work item of their level operators, so other lanes' launches
 * can run between the work items), "serve_priority" (serving lanes created
 * afterwards: 0, default, equal stream priorities; 1: priority grows as the
 * model shrinks, shortest solves first: with serve_persistent = 0 small
 * models' latency under load halves while the largest models wait longer),
 * "spmv32_shape" (launch shape of the FP32 SpMV of MSG_PCG_SOLVE_MIXED on
 * large matrices: 0, default, 4 slots per load group and 8 slices per CTA;
 * 1: 8 and 8; 2: 4 and 4; 3: 8 and 4; results are identical),
 * "tensor_operator" (0, default: every element product in the element's Walsh
 * modes on the FP32 cores; 1: the multigrid loop's level-0 search-direction
 * launch forms E_e Khat u_e on the tensor cores, tcgen05.mma in TF32 with a
 * three-term split; systems without a mass term), "element_batch" (mixed
 * Monte Carlo batches on meshes that are not cube lattices: 1, default, every
 * realization at once through an element-by-element operator over each
 * element's stiffness at E = 1 (FP32 PCG, FP64 iterate and true
 * residuals); 0: realization by realization through the assembled FP32-value
 * PCG of MSG_PCG_SOLVE_MIXED), "element_groups" (launch shape of that
 * element-by-element operator: realization groups of 32 per CTA, each element
 * row block loaded once for all of them; 0, default: the largest of 4, 2, 1
 * dividing the padded group count; 8 is allowed; results are identical),
 * "newmark_predictor" (MSG_NEWMARK_BATCH: 1, default, each step's solve
 * starts from the Newmark predictor u + dt v + (1/2 - alpha) dt^2 a; 0: from
 * the last displacement), "ragged_lattice_loop" (MSG_MC_SOLVE_RAGGED: 1, default, structured cube
 * lattices of the batch are solved by the lattice loop of
 * MSG_MC_SOLVE_BATCH, the other systems together in the element-by-element
 * batch; 0: every system in the element-by-element batch),
 * "ragged_side_by_side" (MSG_MC_SOLVE_RAGGED: 1, default, the lattice loops
 * side by side on their own streams alongside the element-by-element batch;
 * 0: one after another, then the element-by-element batch; the same results).
 * Batched realization counts are padded to a multiple of 64.
 * In the multigrid loop t[5] below is the duration of one search-direction +
 * operator launch and t[6] that of one whole iteration. */
int MSG_SET_OPTION(MSG_CTX ctx, const char* key, double value);
/* The current value of an MSG_SET_OPTION key (MSG_ERR_INVALID_ARGUMENT for an
 * unknown key), or of the read-only keys "memory_used" (device bytes charged
 * to the context), "memory_budget" (its budget, 0 = none) and
 * "device_free_memory" (free bytes on the context's device). */
int MSG_GET_OPTION(MSG_CTX ctx, const char* key, double* value);

/* Kernel launch counter of this context (kernels launched since creation),
 * and device timings in ms (t8 may be NULL):
 * t[0]=KL field, t[1]=inner FP32 loop, t[2]=number of FP64 true-residual
 * (reliable) updates of the last mixed batch, t[3]=FP64 residual steps,
 * t[4]=whole last MC batch (last call); t[5]=mean duration of one
 * matrix-free operator launch, t[6]=mean duration of one inner update launch,
 * t[7]=number of samples behind t[5..6] (one per inner graph launch, CUDA
 * events captured around the first operator/update of each launch, accumulated
 * since the context was created or MSG_STATS_RESET). No reference counterpart
 * (the reference writes stopwatch times to text files,
 * MonteCarloAnalyzerWithStochasticMaterial.cs:244-292). */
int MSG_STATS(MSG_CTX ctx, int64_t* launches, double* t8);
int MSG_STATS_RESET(MSG_CTX ctx);

/* Self-test of the failure path of the bounded device waits (no reference
 * counterpart). Every wait of the staged operators (an mbarrier that a TMA
 * load or the other warps complete) polls a bounded number of times and, when
 * it gives up, records the expiry in an error word and lets its kernel return;
 * the batch then ends with MSG_ERR_TIMEOUT and the context stays usable. This
 * entry launches one thread that waits, with `polls` polls (1 ... 2^24), on an
 * mbarrier that nothing completes: it returns MSG_ERR_TIMEOUT when the wait
 * expired as designed (MSG_OK would mean it completed). */
int MSG_WAIT_SELFTEST(MSG_CTX ctx, int64_t polls);

#ifdef __cplusplus
}
#endif
#endif
