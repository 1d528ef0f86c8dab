/*
 * CPU oracle for the MSolve Hexa8 linear-elastic solve path.
 *
 * TEST INFRASTRUCTURE ONLY. This library restates, in plain C++ FP64, the
 * algorithms of the reference (isaar/MSolve, C# + Fortran) on the Hexa8 static
 * solve and Monte Carlo realization path. It exists to check the CUDA product
 * library and to time a CPU baseline. Only tests/, __graft_entry__.smoke() and
 * bench.py (cpu_baseline leg and --impl reference) may load it; the product
 * (msolve_b200, libmsolve_gpu.so) never links or calls it.
 *
 * Parity status: the reference cannot be compiled or run on this machine
 * (C#/.NET 4 and Intel Fortran; no dotnet/mono/gfortran present), and it ships
 * no tests, fixtures or golden vectors. Parity is therefore UNPINNED against
 * reference execution. The restatement is pinned instead by known-answer tests
 * that do not depend on this code: the closed-form (exact rational) unit-cube
 * Hexa8 stiffness, agreement of the Fortran-path and C#-path restatements,
 * rigid-body null space, patch tests and direct-vs-iterative agreement.
 *
 * Every function cites the reference file:line it restates (paths relative to
 * the MSolve project root).
 */
#ifndef MSOLVE_ORACLE_H
#define MSOLVE_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- element level (FEMElements/FEMElements/rElHexa8.f90, Hexa8.cs) ---- */
void orc_elastic_D(double E, double nu, double* D36);
int orc_h8_gauss_matrices(const double* xyz24, double* weight8, double* S64, double* DS192,
                          double* J72, double* detJ8, double* B1152);
void orc_h8_k(const double* Emat288, const double* B1152, const double* weight8, double* K300);
int orc_h8_stiffness_fortran(const double* xyz24, double E, double nu, double* K300);
int orc_h8_stiffness_csharp(const double* xyz24, double E, double nu, double* K300);
int orc_h8_consistent_mass(const double* xyz24, double rho, double* M300);
void orc_h8_stiffness_batch(int n, const double* xyz, const double* E, double nu, double* K, int* status);
void orc_h8_strains(const double* B1152, const double* u24, double* strains48);
int orc_h8_stress(const double* xyz24, double E, double nu, const double* u24, const double* du24,
                  double* strains48, double* stresses48, double* forces24);
void orc_h8_stress_batch(int n, const double* xyz, const double* E, double nu, const double* u, const double* du,
                         double* strains, double* stresses, double* forces, int* status);

int orc_pcg_reorth_csr(int n, const int64_t* rp, const int* ci, const double* v, const double* b, double* x,
                       double* P, double* Q, double* pq, int cap, int* count, int start, int max_it, double tol,
                       int* iterations, double* rel_res);
int orc_pc_size(int m, int p);
int orc_pc_basis(int m, int p, int* basis, int* norms);
void orc_pc_gaussian_matvec(int n, const int64_t* rp, const int* ci, const double* vals, int64_t nnz, int m, int p,
                            const double* u, double* y);
void orc_kl_field_gaussian(int ne, const double* cen, const double* L, int K, const double* w3, const double* amp3,
                           const int* idx3, const double* eig, int R, const double* xi, double mean, double cov,
                           double* E);

/* ---- mesh / DOFs / loads (Hexa8MeshGenerator.cs, Model.cs, Subdomain.cs) ---- */
void orc_block_nodes(int nx, int ny, int nz, double h, double* xyz);
void orc_block_conn(int nx, int ny, int nz, int* conn);
int orc_enumerate_dofs(int n_nodes, const uint8_t* constrained3, int* dof3);

/* ---- skyline (GlobalMatrixAssemblerSkyline.cs, SkylineMatrix2D.cs) ---- */
int64_t orc_skyline_rowindex(int n_elems, const int* conn, const int* dof3, int n_dofs, int64_t* rowIndex);
void orc_skyline_assemble(int n_elems, const int* conn, const int* dof3, const double* Ke300,
                          const int64_t* rowIndex, double* data);
int orc_skyline_factorize(int n_dofs, const int64_t* rowIndex, double* data, double tol, int* n_zems);
void orc_skyline_solve(int n_dofs, const int64_t* rowIndex, const double* data, const double* f, double* x);
void orc_skyline_multiply(int n_dofs, const int64_t* rowIndex, const double* data, const double* x, double* y);

/* ---- CSR (assembled restatement of the skyline sum for sizes skyline cannot hold) ---- */
int64_t orc_csr_pattern(int n_nodes, int n_elems, const int* conn, const int* dof3, int n_dofs,
                        int64_t* rowptr, int* colind);
void orc_csr_assemble(int n_elems, const int* conn, const int* dof3, const double* Ke300,
                      const int64_t* rowptr, const int* colind, double* val);
void orc_csr_multiply(int n, const int64_t* rowptr, const int* colind, const double* val,
                      const double* x, double* y);

/* ---- PCG (PCG/SolverPCG.cs + SolverPCGSimpleSearchVectorCalculator.cs) ---- */
int orc_pcg_csr_jacobi(int n, const int64_t* rowptr, const int* colind, const double* val,
                       const double* b, double* x, int max_it, double tol,
                       int* iterations, int* matvecs, double* rel_res);
int orc_pcg_skyline(int n, const int64_t* rowIndex, const double* data, const double* precond_ldlt,
                    const double* b, double* x, int max_it, double tol,
                    int* iterations, int* matvecs, double* rel_res);

/* ---- Karhunen-Loeve lognormal field (LognormalFileStochasticCoefficientsProvider.cs) ---- */
int orc_kl_1d_modes(double half_length, double corr_len, int n_modes, double* w, double* amp, double* lam);
int orc_kl_table(const double* domain3, double corr_len, int n_terms, int n1d,
                 double* w3, double* amp3, int* idx3, double* eig);
void orc_kl_field(int n_elems, const double* centroids, const double* domain3, int n_terms,
                  const double* w3, const double* amp3, const int* idx3, const double* eig,
                  int n_real, const double* xi, double mean, double sigma, int mean_correction,
                  double* E);

/* ---- structured-block helpers used by the Monte Carlo and Newmark restatements ---- */
int orc_block_solve_pcg(int nx, int ny, int nz, double h, const uint8_t* constrained3,
                        const double* E_elem, double nu, const double* b_dof,
                        double* x_dof, int max_it, double tol, int* iterations, double* rel_res);

int orc_block_newmark(int nx, int ny, int nz, double h, const uint8_t* constrained3, const double* E_elem, double nu,
                      double rho, double ray_alpha, double ray_beta, double nm_alpha, double nm_delta, double dt,
                      int n_steps, double acc_amp, double acc_period, int acc_dir, const double* f_static, int solver,
                      double tol, int tip_dof, double* tip_hist, double* u_final, int* total_its);

/* Realizations in parallel, one per OpenMP thread (E [R][ne], x [R][N]). */
void orc_block_solve_pcg_batch(int R, int nx, int ny, int nz, double h, const uint8_t* constrained3, const double* E,
                               double nu, const double* b, double* x, int N, int max_it, double tol, int* status,
                               int* iterations, double* rel_res);
void orc_block_newmark_batch(int R, int nx, int ny, int nz, double h, const uint8_t* constrained3, const double* E,
                             double nu, double rho, double ray_alpha, double ray_beta, double nm_alpha,
                             double nm_delta, double dt, int n_steps, double acc_amp, double acc_period, int acc_dir,
                             const double* f_static, int solver, double tol, int tip_dof, int N, double* tip_hist,
                             double* u_final, int* total_its, int* status);

int orc_num_threads(void);

#ifdef __cplusplus
}
#endif
#endif
