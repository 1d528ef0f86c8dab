// Internal declarations shared by the host runtime (msg_api.cpp) and the
// CUDA kernels (*.cu) of libmsolve_gpu.so.
#pragma once

#include <nvtx3/nvToolsExt.h>
#include <cuda_runtime.h>

#include <atomic>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <memory>
#include <functional>
#include <mutex>
#include <string>
#include <vector>

#include "msolve_gpu.h"

namespace msg {

// Packed row-wise upper index of a 24x24 symmetric matrix (SymmetricMatrix2D.IndexOf).
__host__ __device__ inline int packed_index(int i, int j) {
  int r = i < j ? i : j, c = i < j ? j : i;
  return r * (47 - r) / 2 + c;
}

// Hexa8 local corner numbering of (ax, ay, az) in {0,1}^3 (rElHexa8.f90:43-68).
__host__ __device__ constexpr int corner_id(int ax, int ay, int az) {
  return az * 4 + (ay ? (ax ? 2 : 3) : (ax ? 1 : 0));
}

constexpr int kGmgMaxLevels = 6;  // multigrid lattice levels at most (fine level included)
constexpr int kWorkSlots = 40;    // context workspace slots (see workspace())

struct Context;

// Device allocation charged against the context's memory budget.
struct DevMem {
  void* ptr = nullptr;
  size_t bytes = 0;
  Context* ctx = nullptr;
  DevMem() = default;
  DevMem(const DevMem&) = delete;
  DevMem& operator=(const DevMem&) = delete;
  ~DevMem();
  int alloc(Context* c, size_t n);
  void release();
  template <class T> T* as() const { return static_cast<T*>(ptr); }
};

// Handles are reference counted: a mesh holds its context, a matrix holds its
// mesh, so the caller may destroy them in any order (a garbage-collected host
// such as .NET finalises in arbitrary order); the object is freed with its
// last reference.
struct LatticeRunner;

struct Context {
  std::atomic<int> refs{1};
  int device = 0;
  cudaStream_t stream = nullptr;
  uint64_t budget = 0;           // 0 = unlimited
  std::atomic<uint64_t> used{0};
  std::recursive_mutex mu;
  std::string last_error;
  std::mutex err_mu;  // last_error: a ragged batch's lattice loops run on a second host thread
  std::atomic<int64_t> launches{0};
  double t_phase[5] = {0, 0, 0, 0, 0};
  // live per-launch samples of the inner operator / update kernels (event
  // records captured in the inner-loop graph): sum of ms and sample count
  double op_ms_sum = 0, upd_ms_sum = 0;
  int64_t op_samples = 0;
  int sm_count = 148;
  // mixed-solver tunables (MSG_SET_OPTION)
  double reliable_delta = 0.1;  // FP64 residual replacement when ||r|| drops by this factor
  int chunk = 16;               // inner iterations per captured graph launch
  int fixed_updates = 0;        // 1: FP64 true-residual step after every graph chunk (batch-invariant results)
  // multigrid preconditioner of the batched lattice solves
  // 1: V-cycle preconditioned loop for systems without a mass term, 2: also with
  // one, 0: Jacobi loop (the V-cycle needs a lattice that coarsens at least once)
  int multigrid = 1;
  int mg_levels = kGmgMaxLevels; // lattice levels at most, fine level included (2..kGmgMaxLevels)
  int mg_sweeps = 20;           // damped Jacobi sweeps on the coarsest level
  double mg_omega = 0.0;        // Jacobi damping; 0 = from the element stiffness
  double mg_delta = 1e-3;       // reliable-update factor of the V-cycle-preconditioned loops
  int mg_packed = 1;            // 1: level-0 operator with two realizations per lane (packed FP32)
  int mg_fused_coarse = 1;      // 1: all coarsest-level sweeps in one launch (when the level fits a CTA)
  int tensor_op = 0;            // 1: the multigrid loop's level-0 search-direction launch on the tensor cores
  int spmv32_shape = 0;         // launch shape of the mixed assembled loop's FP32 SpMV (slots per group, slices per CTA)
  int element_batch = 1;        // mixed mode on non-lattice meshes: 1 batched element-by-element loop, 0 per realization
  int element_groups = 0;       // realization groups of 32 per CTA of the element-by-element FP32 operator (0 auto)
  int ragged_lattice_loop = 1;  // ragged batches: cube lattices through the lattice loop (1) or the shared loop (0)
  int ragged_side_by_side = 1;  // ragged batches: the cube lattices' loops side by side (1) or one after another (0)
  int nm_predictor = 1;         // Newmark steps start from the Newmark predictor (1) or the last displacement (0)
  int serve_persistent = 1;     // serving lanes: 1 persistent grids, 0 one CTA per work item
  int serve_priority = 0;       // serving lanes: 1 stream priority grows as the model shrinks, 0 all equal
  // Workspace kept across calls (allocation and cudaFree synchronise the
  // device; a batch reuses the previous batch's buffers when they are large
  // enough). Slots are owned by the call sites that use them.
  DevMem* work[kWorkSlots] = {nullptr};
  // lattice buffer sets (kWorkSlots each) of the V-cycle preconditioners of an
  // element-by-element batch with several of them: set k for the k-th such
  // system, kept (and grown) across calls like the workspace slots
  std::vector<DevMem*> vc_pool;
  // the ragged batch's cube lattices, solved side by side: runner k (a stream,
  // 12 events, the loop graph and a lattice buffer set) serves the k-th of them,
  // kept across calls
  std::vector<LatticeRunner*> lat_runners;
  // per-context host/driver resources reused by every batch (created lazily)
  int* h_flags = nullptr;           // 4 KB of pinned host memory, mapped into the device
  int* d_hflags = nullptr;          // the device's address of h_flags
  double* h_stage = nullptr;        // 8 KB of pinned host memory: small uploads issued as true async copies
  // unit-cube element matrices already computed (kind 0: stiffness at E = 1
  // for (h, nu); 1: consistent mass for (h, rho)): later batches read no
  // device data and free no device memory while setting up
  struct CubeMatrix {
    int kind;
    double h, param;
    double v[576];
  };
  std::vector<CubeMatrix> cube_cache;
  std::mutex cube_mu;
  cudaEvent_t ev[14] = {nullptr};   // timing events
  // pipelined Monte Carlo batches: the displacement copy to the host of one
  // call runs on copy_stream from output buffer pipe_next ^ 1 while the next
  // call computes into the other buffer
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t pipe_ev[2] = {nullptr, nullptr};  // copy of buffer i done
  cudaEvent_t pipe_ready = nullptr;             // batch done, its copy may start
  bool pipe_pending[2] = {false, false};
  int pipe_next = 0;
  cudaGraphExec_t batch_graph = nullptr;  // inner-loop graph of the last batch configuration
  size_t batch_graph_key = 0;
  void* server = nullptr;  // serving worker and lanes (serve.cpp), nullptr until MSG_SERVE_START
  // FP64 Monte Carlo drop-in: the assembled matrix, its element-matrix scratch and
  // staging kept across calls for one mesh (weak: dropped when that mesh is freed)
  struct Matrix* mc_matrix = nullptr;
  DevMem* mc_ke = nullptr;
  DevMem* mc_st = nullptr;
  DevMem* mc_E = nullptr;
  // device address of MSG_PCG_SOLVE_NOALLOC's fixed scratch array on this
  // context's device, looked up by MSG_CREATE (noalloc_scratch_address)
  unsigned char* noalloc_scratch = nullptr;
  ~Context();
};

// Device address of MSG_PCG_SOLVE_NOALLOC's scratch array on the current device
// (kernels_bsr.cu); MSG_CREATE calls it with the context's device current.
cudaError_t noalloc_scratch_address(unsigned char** out);

// Stop the serving worker of a context and free its lanes (serve.cpp).
void server_destroy(Context* ctx);

// Lazily created pinned flags and events of a context.
int context_resources(Context* ctx);

// Workspace slot `slot` of at least `bytes` bytes (grown, never shrunk).
int workspace(Context* ctx, int slot, size_t bytes, void** out);
// Waits for every displacement copy of the pipelined batches still in flight.
int pipe_flush(Context* ctx);
// h_host[0 .. n) = d_src[0 .. n) on stream st, written by a one-block kernel
// when d_hmapped (the device address of h_host) is given and n <= 1024, so that the read
// never waits behind copies in flight on the device's copy engines; a copy
// otherwise. Read h_host after synchronizing st.
int publish_flags(Context* ctx, const int* d_src, int n, int* h_host, int* d_hmapped, cudaStream_t st);

void retain(Context* ctx);
void release(Context* ctx);
struct Mesh;
void retain(Mesh* m);
void release(Mesh* m);

int set_error(Context* ctx, int code, const char* fmt, ...);
int cuda_error(Context* ctx, cudaError_t e, const char* where);

#define MSG_CUDA(ctx, call)                                   \
  do {                                                        \
    cudaError_t _e = (call);                                  \
    if (_e != cudaSuccess) return ::msg::cuda_error((ctx), _e, #call); \
  } while (0)

#define MSG_TRY(call)            \
  do {                           \
    int _s = (call);             \
    if (_s != MSG_OK) return _s; \
  } while (0)

// Kernels launched counter (the bench reports how many of this library's
// kernels ran inside its timed region).
inline void count_launch(Context* ctx, int n = 1) { ctx->launches += n; }

// Host-side NVTX range (NVTX v3, header-only: a no-op unless a tool is attached)
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};

// 3x3-block sliced-ELL (SELL-32) pattern of the global stiffness over all
// mesh nodes. Block row = node. Slices of 32 rows; slot s of slice z holds
// one block column per row. Layouts: col[(slot_base + s)*32 + lane],
// val[((slot_base + s)*9 + k)*32 + lane] with k = 3*row_comp + col_comp.
struct BlockPattern {
  int n_rows = 0;                       // nodes
  int n_slices = 0;
  int64_t n_slots = 0;                  // total slots (each 32 lanes)
  int64_t nnzb = 0;                     // true blocks
  std::vector<int64_t> slice_ptr;       // n_slices + 1, in slots
  std::vector<int> col;                 // n_slots*32, -1 = padding
  std::vector<int> diag_pos;            // per row: flat lane position of its diagonal block
  // assembly contributions: per flat position, list of (e*64 + a*8 + b)
  std::vector<int64_t> contrib_ptr;     // n_slots*32 + 1
  std::vector<int> contrib;
};

struct Mesh {
  std::atomic<int> refs{1};
  Context* ctx = nullptr;
  int n_nodes = 0, n_elems = 0, n_dofs = 0;
  std::vector<double> xyz;   // [n_nodes][3]
  std::vector<int> conn;     // [n_elems][8]
  std::vector<int> dof;      // [n_nodes][3]
  BlockPattern pat;
  // structured cube lattice (generator order) -> matrix-free batched path
  bool structured = false;
  int nx = 0, ny = 0, nz = 0;
  double h = 0, origin[3] = {0, 0, 0};
  // device copies
  DevMem d_exyz;       // [n_elems][24] element coordinates
  DevMem d_dof;        // [n_nodes][3]
  DevMem d_conn;       // [n_elems][8]
  DevMem d_col, d_slice_ptr, d_contrib_ptr, d_contrib, d_diag_pos;
  DevMem d_mask;       // [n_nodes] uint8 bit c = component c constrained
  DevMem d_centroid;   // [n_elems][3]
  DevMem d_free_rows;  // [n_dofs] int: node*3+c for each free DOF (DOF -> node layout)
  // padded lattice of a structured mesh (one ghost node layer per side):
  // NXp = nx+3 nodes per x row etc.; element (i,j,k) is stored at the padded
  // node of its lower corner, so nodes and elements share one index space.
  int NXp = 0, NYp = 0, NZp = 0;
  DevMem d_pad_free_rows;  // [n_dofs] padded node*3 + c
  DevMem d_pad_elem_row;   // [n_elems] padded row of the element
  DevMem d_pad_mask;       // [padded nodes] constrained bits, ghosts = 7
  DevMem d_pad_interior;   // [interior nodes] padded index of interior node t (generator order)
  // coarse lattices of the multigrid preconditioner, level l = 1..gmg_levels-1
  // (node (i, j, k) of level l sits on fine node 2^l (i, j, k)): constrained
  // bits of the padded nodes (ghosts 7) and the interior list; built on first use
  std::mutex gmg_mu;
  int gmg_levels = 1;
  DevMem d_gmg_mask[kGmgMaxLevels], d_gmg_interior[kGmgMaxLevels];
  // lattice topology with moved nodes (the generator's numbering and element
  // order, any coordinates; not `structured`): the element-by-element loop
  // takes the multigrid V-cycle of the cube lattice of the same numbering
  // (`shadow`, built on first use, owned) as its preconditioner
  bool topo_lattice = false;
  int tnx = 0, tny = 0, tnz = 0;
  Mesh* shadow = nullptr;
  std::mutex shadow_mu;
};

struct PcgState {
  double zr, pq, rr, bnorm, alpha, beta, err;
  // need (mixed precision) follows done: the host reads both as one pair
  int it, done, need, status, iterations, matvecs, max_it;
  double tol;
  unsigned int counter;
  // mixed precision (FP32 matrix values and vectors, FP64 iterate): the loop
  // pauses (need = 1) when the recursive residual has dropped by delta since
  // err_ref or below tol, and the host replaces it with the FP64 true residual
  double delta, err_ref;
  int mixed;
  // rounds of the graph's device loop (chunks of iterations) and the FP64
  // true-residual pauses among them
  int rounds, pauses, pad;
};

struct Matrix {
  Mesh* mesh = nullptr;
  DevMem d_val;   // SELL values FP64
  DevMem d_val32; // SELL values FP32 (mixed-precision solves; built on first use)
  DevMem d_bn, d_xn, d_bd;  // node-layout b and x, DOF-layout staging of the host entry points
  DevMem d_dinv;  // [n_nodes*3]
  // PCG workspace (node layout, 3 per node)
  DevMem d_r, d_p0, d_p1, d_q, d_partial, d_state, d_tmp, d_tmp2;
  DevMem d_m32;  // mixed loop: FP32 r, q, d and D^-1 ([4][n_nodes*3]; p32 in d_tmp2)
  cudaGraphExec_t graph = nullptr;
  int graph_chunk = 0;
  int graph_mixed = 0;
  const void* graph_x = nullptr;  // output vector the captured graph writes (not owned)
  const void* graph_b = nullptr;  // right-hand side its true-residual steps read (not owned)
  ~Matrix();
};

// Search vectors (p, K p) kept across solves for the re-orthogonalised PCG
// (kernels_recycle.cu): node layout, count pairs of capacity in use.
struct SearchVectorStore {
  Mesh* mesh = nullptr;
  int64_t n3 = 0;
  int capacity = 0, count = 0;
  DevMem P, Q, pq, coef, work, scal;
  ~SearchVectorStore() {
    if (mesh) release(mesh);
  }
};
int svs_create(Context* ctx, Mesh* m, int capacity, SearchVectorStore** out);
int pcg_reorth_solve(Context* ctx, Matrix* A, SearchVectorStore* S, const double* d_b, double* d_x, int start_mode,
                     int max_it, double tol, int* iterations, double* rel_res);

// Polynomial chaos (pc.cpp): size of the basis of m Gaussian variables up to
// degree p, the basis in the reference's order with its squared norms, and the
// Galerkin terms of each output block (CSR over blocks: matrix, input block, weight).
int pc_size(int m, int p);
int pc_basis(int m, int p, std::vector<int>& basis, std::vector<int>& norms);
int pc_gaussian_terms(int m, int p, std::vector<int>& term_ptr, std::vector<int>& term_pos, std::vector<int>& term_k,
                      std::vector<double>& term_c);
// y = Galerkin product of the block vector u [P][n_dofs] (host), kernels_block.cu
int pc_matvec(Context* ctx, Mesh* m, double nu, const MSG_KL* kl, int mo, int po, const double* u_host,
              double* y_host);

// ---------------------------------------------------------------- kernel launchers (kernels_*.cu)
int launch_h8_ke(Context* ctx, int n, const double* d_xyz, const double* d_E, double E_scalar, double nu,
                 double* d_K, int* d_status);
int launch_h8_me(Context* ctx, int n, const double* d_xyz, double rho, double* d_M, int* d_status);
// Strains, stresses (per Gauss point) and internal forces of n element instances
// (instance i = element i % n_e of realization i / n_e); displacements from
// d_u [n][24] or gathered from d_X [R][n_dofs] through d_conn/d_dof.
int launch_h8_stress(Context* ctx, int n, const double* d_xyz, const double* d_E, double E_scalar, double nu,
                     const double* d_u, const double* d_du, const double* d_X, const int* d_conn, const int* d_dof,
                     int n_e, int n_dofs, double* d_strains, double* d_stresses, double* d_forces, int* d_status);
int launch_bsr_assemble(Context* ctx, const Mesh* m, const double* d_Ke, double* d_val);
int launch_bsr_diag_inv(Context* ctx, const Mesh* m, const double* d_val, double* d_dinv);
int launch_bsr_spmv(Context* ctx, const Mesh* m, const double* d_val, const double* d_x, double* d_y);
int launch_dof_to_node(Context* ctx, const Mesh* m, const double* d_in, double* d_out, int n_vec, int64_t in_stride,
                       int64_t out_stride);
int launch_node_to_dof(Context* ctx, const Mesh* m, const double* d_in, double* d_out, int n_vec, int64_t in_stride,
                       int64_t out_stride);
// FP32 copy b[0..n) of FP64 a on the context's stream.
int launch_to_f32(Context* ctx, size_t n, const double* a, float* b);
// mixed: FP32 matrix values and vectors in the loop, the iterate in FP64, FP64
// true-residual replacement (reliable updates), stop on the FP64 true residual.
int pcg_solve_device(Context* ctx, Matrix* A, const double* d_b_node, double* d_x_node, int max_it, double tol,
                     int* iterations, double* rel_res, int* status, bool mixed = false);

// KL field: E64/E32 [n_elems][Rp] (realization innermost) and/or E64 [R][n_elems].
struct KLDevice {
  int n_terms = 0;
  double* psi = nullptr;  // [K][n_elems], context workspace slot 15
  double mu = 0;
  int gaussian = 0;       // 1: E = mean (1 + sum xi psi); 0: E = exp(mu + sum xi psi)
  double mean = 1.0;
};
int kl_prepare(Context* ctx, const Mesh* m, const MSG_KL* kl, KLDevice* out);
// d_elem_row (nullable): output row of element e in the [row][Rp] layouts.
int launch_kl_field(Context* ctx, const Mesh* m, const KLDevice* kl, int R, int Rp, const double* d_xi,
                    double* d_E64_er, float* d_E32_er, double* d_E64_re, const int* d_elem_row = nullptr);

// E of a list of realization slots into the padded [row][Rp] layouts (FP64 and FP32)
int launch_kl_field_slots(cudaStream_t st, const Mesh* m, const KLDevice* kl, int n_slots, const int* d_slots,
                          const double* d_xi, int Rp, double* d_E64, float* d_E32);

// self-test of the bounded device waits (kernels_block.cu): *expired = 1 when the wait gave up
int wait_selftest(Context* ctx, long polls, int* expired);

// batched mixed-precision solve on a structured lattice (kernels_block.cu)
struct BatchOut {
  double* tip = nullptr;
  int* iterations = nullptr;
  double* rel_res = nullptr;
};
int block_mixed_solve(Context* ctx, Mesh* m, double nu, const KLDevice* kl, const double* d_xi, int R, int Rp,
                      const double* d_b_dof, int max_it, double tol, int tip_dof, double* d_X, BatchOut out);

// The cube lattice with the numbering of a lattice-topology mesh (built once;
// a cube lattice is its own).
int lattice_shadow(Context* ctx, Mesh* m, Mesh** out);
// Multigrid V-cycle of a cube lattice mesh as a preconditioner of another
// operator with the same node numbering (kernels_block.cu): R realizations of
// the KL field xi [R][n_terms] (on the lattice's element centroids), Rp a
// multiple of 32. apply enqueues z = V(r) on st for node-layout FP32 vectors
// [n_nodes * 3][Rp] (constrained components of r zero); graph-capturable.
// own: kWorkSlots lattice buffers for this preconditioner (several
// preconditioners at once; not owned, kept by the caller across calls), or
// nullptr for the context's workspace. r_node nullptr: r is already in the
// lattice's r buffer; z_node nullptr: z stays in the lattice's z buffer.
int gmg_precond_create(Context* ctx, Mesh* lattice, double nu, const MSG_KL* kl, const double* d_xi, int R, int Rp,
                       DevMem* own, void** out);
int gmg_precond_apply(Context* ctx, void* P, const float* r_node, float* z_node, cudaStream_t st);
// The lattice's r and z buffers ((padded node * 3 + c) * Rp + realization), the
// padded index of each mesh node and the buffers' Rp; the partials of z.r of the
// last apply (zr_blocks blocks: zr_part[(block * Rp + realization) * 2]).
void gmg_precond_buffers(void* P, float** r_lat, float** z_lat, const int** node_to_lattice, int* Rp,
                         const double** zr_part, int* zr_blocks);
void gmg_precond_destroy(void* P);

// One system of a batched element-by-element solve (kernels_ebe.cu): a mesh
// of any shape with its material, KL field and realizations; xi [R][n_terms],
// b [n_dofs] and X [R][n_dofs] on the device (X may be null), tip, iterations
// and residuals [R] on the host (each may be null).
struct RgInput {
  Mesh* m = nullptr;
  double nu = 0.3;
  const MSG_KL* kl = nullptr;
  int R = 0;
  const double* d_xi = nullptr;
  const double* d_b = nullptr;
  double* d_X = nullptr;
  double* h_tip = nullptr;
  int tip_dof = -1;
  int* h_its = nullptr;
  double* h_res = nullptr;
};
// All realizations of all systems in one loop (each system's realizations
// padded to 32 inside); a system's results independent of the other systems.
int ebe_ragged_solve(Context* ctx, const std::vector<RgInput>& in, int max_it, double tol);
// PCG over the element-by-element operator for every system of a batch, each
// preconditioned by the multigrid V-cycle of its cube lattice (use_vcycle[i])
// or by the diagonal; standard PCG, two iterations to a graph launch.
int ebe_mg_solve(Context* ctx, const std::vector<RgInput>& in, const std::vector<int>& use_vcycle, int max_it,
                 double tol);
// The element-by-element batch: systems whose mesh has the lattice's numbering
// and coarsens take the V-cycle (multigrid option != 0; then ebe_mg_solve for
// the whole batch), a batch without one the fused Jacobi loop (ebe_ragged_solve).
int ebe_solve(Context* ctx, const std::vector<RgInput>& in, int max_it, double tol);

// Newmark batch (implicit integration of every realization, constant time step)
struct NewmarkParams {
  double rho = 1.0;                        // density of the consistent mass
  double ray_alpha = 0.0, ray_beta = 0.0;  // Rayleigh damping C = ray_alpha M + ray_beta K
  double alpha = 0.25, delta = 0.5;        // Newmark parameters (NewmarkDynamicAnalyzer alpha, delta)
  double dt = 0.01;
  int n_steps = 0;
  double acc_amp = 0.0, acc_period = 1.0;  // ground acceleration acc_amp sin(2 pi t / acc_period)
  int acc_dir = 0;                         // 0 x, 1 y, 2 z
};
int block_newmark(Context* ctx, Mesh* m, double nu, const KLDevice* kl, const double* d_xi, int R, int Rp,
                  const NewmarkParams& nm, const double* d_f_dof, int max_it, double tol, int tip_dof,
                  double* tip_hist, double* d_U, int* its_total);

// Cube-lattice batches solved side by side (kernels_block.cu): the ragged
// batch's lattices, each with the outputs of MSG_MC_SOLVE_BATCH_DEVICE (X and
// the tip on the device and the host, iterations and residuals on the host);
// status is each batch's outcome.
struct LatticeJob {
  Mesh* m = nullptr;
  double nu = 0.0;
  const MSG_KL* kl = nullptr;
  const double* d_xi = nullptr;
  const double* d_b = nullptr;
  int R = 0, tip_dof = -1;
  double* d_X = nullptr;
  double* h_tip = nullptr;
  int* h_its = nullptr;
  double* h_res = nullptr;
  int status = 0;
};
struct LatticeRunner {
  cudaStream_t st = nullptr;
  cudaEvent_t ev[12] = {};
  cudaGraphExec_t graph = nullptr;
  size_t graph_key = 0;
  DevMem* pool = nullptr;  // kWorkSlots buffers
  DevMem tip;              // the tip displacement of every realization
  ~LatticeRunner();
};
// alongside (optional) runs on the calling thread while a second host thread
// steps the lattices' loops; its status is returned when theirs is MSG_OK.
int block_mixed_solve_many(Context* ctx, std::vector<LatticeJob>& jobs, int max_it, double tol,
                           const std::function<int()>& alongside);

// Serving lanes (kernels_block.cu): continuous batching of one model's requests.
struct Lane;
int lane_create(Context* ctx, Mesh* m, double nu, const MSG_KL* kl, const double* b_host, int capacity, double tol,
                int max_it, Lane** out);
void lane_destroy(Lane* L);
int lane_capacity(const Lane* L);
int lane_n_dofs(const Lane* L);
int lane_n_terms(const Lane* L);
void lane_stage(Lane* L, int slot, const double* xi);
int lane_abort(Lane* L, int slot);
int lane_cycle(Lane* L, int* state, int* its, double* res, int* n_active);
int lane_fetch(Lane* L, int slot, double* X);

// Element stiffness of one cube of side h at E=1 (host, via the K1 kernel): K[24][24] full.
int unit_cube_khat(Context* ctx, double h, double nu, double* K576);
// Consistent mass of one cube of side h and density rho (host, via the mass kernel): M[24][24] full.
int unit_cube_mhat(Context* ctx, double h, double rho, double* M576);

}  // namespace msg

struct msg_context : msg::Context {};
struct msg_mesh : msg::Mesh {};
struct msg_matrix : msg::Matrix {};
struct msg_svs : msg::SearchVectorStore {};
