// Batched mixed-precision Monte Carlo solve on a structured cube lattice.
//
// The path of MonteCarloAnalyzerWithStochasticMaterial.SolveNormal
// (ISAAR.MSolve.Analyzers/MonteCarloAnalyzerWithStochasticMaterial.cs:232-296),
// restated for all realizations at once. For a lattice of equal cubes every
// element stiffness is K_e = E_e * Khat (Hexa8WithStochasticMaterial.cs:61-110
// evaluates E once at the centroid), so the global operator is applied
// matrix-free: y_n = sum_{e owns n} E_e * Khat[rows of n] . u_e.
//
// Layout (realization innermost, padded lattice): a batch vector is
// v[(node*3 + comp)*Rp + r] over a lattice with one ghost node layer on every
// side (node = I + NXp*(J + NYp*K), interior I = 1..nx+1); element (i,j,k) is
// stored at the padded index of its lower-corner node, ghost elements hold E=0.
// Ghost entries of every vector stay zero, so the stencil needs no bounds
// checks. A warp is 32 realizations of one node: every access is one coalesced
// 128-byte line and per-realization dot products need no cross-lane reduction.
//
// Operator kernels (k_op_modal, k_lvl_op, k_lvl_op2, k_resid_modal): a CTA owns
// a tile of node pencils along x and walks the x-planes, staging each plane's
// patch with TMA; the element product is applied in the element's Walsh modes
// (below), and the four elements around a node meet in a shared-memory
// exchange buffer in fixed order. Each output is written once: no atomics;
// results are deterministic and independent of the batch mix. k_lvl_tc applies
// the same product on the tensor cores (option "tensor_operator").
//
// Solvers: the single-reduction FP32 Jacobi-PCG loop (k_op_modal +
// k_alpha_gamma per iteration) and the multigrid-preconditioned loop
// (gmg_iteration), each captured as one CUDA graph of `chunk` iterations, with
// reliable updates in FP64: x += d + alpha p (the pending term), d = 0,
// r = b - K x with the FP64 Walsh-mode operator (k_resid_modal); a true
// ||r||/||b|| < tol ends a realization, otherwise the search direction is kept
// (beta = gamma_new / gamma_prev), so the Krylov progress survives.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <thread>

#include <cuda.h>
#include <cudaTypedefs.h>

#include <utility>

#include "khat_classes.h"

#include "msg_internal.h"

namespace msg {
namespace {

constexpr int kTJ = 2, kTK = 2, kWarps = kTJ * kTK;  // pencils per CTA (2 x 2 in (j,k))

// The unit-cube stiffness as its value classes (khat_classes.h): entry
// (row, col) = sign * v[class], both compile-time constants of (row, col).
template <class T> struct KhatClasses { T v[kKhatClasses]; };
using KhatF = KhatClasses<float>;
using KhatD = KhatClasses<double>;

template <int... Is, class F>
__device__ __forceinline__ void static_for_impl(std::integer_sequence<int, Is...>, F&& f) {
  (f(std::integral_constant<int, Is>{}), ...);
}
// f(std::integral_constant<int, i>) for i = 0..N-1, each index a constant expression
template <int N, class F>
__device__ __forceinline__ void static_for(F&& f) {
  static_for_impl(std::make_integer_sequence<int, N>{}, f);
}

struct Lattice {
  int NX, NY, NZ;     // interior nodes per axis (nx+1 ...)
  int NXp, NYp, NZp;  // padded nodes per axis
  int Rp;             // padded realizations (multiple of 32)
  int tiles_j;        // ceil(NY / kTJ)
  int n_pad;          // NXp*NYp*NZp
  int n_int;          // NX*NY*NZ
};

template <class T> struct KhatOf;
template <> struct KhatOf<float> { using type = KhatF; };
template <> struct KhatOf<double> { using type = KhatD; };

template <class T>
__device__ __forceinline__ T ldv(const T* p) { return __ldg(p); }

// Consistent mass of a cube element as value classes: entry (a, c), (b, c2)
// is delta(c, c2) * v[number of coordinates in which corners a and b differ].
template <class T> struct MassClasses { T v[4]; };

// Contribution of one input plane to one output node through the 4 elements
// of one x-slab: y[c] += E_e * sum_{by,bz,c2} Khat[(an,c),(bn,c2)] * u[ey+by][ez+bz][c2]
// with an = corner(AX, 1-ey, 1-ez) (output node in the element) and
// bn = corner(BX, by, bz) (input node in the element); with kMass also
// + sum_{by,bz} Mhat[an,bn] u[ey+by][ez+bz][c] for every real element (E > 0).
template <class T, int AX, int BX, bool kMass = false>
__device__ __forceinline__ void slab_apply(const T (&kv)[kKhatClasses], const T (&u)[3][3][3], const T (&E)[2][2],
                                           T (&y)[3], const T* mv = nullptr) {
  static_for<2>([&](auto EY) {
    static_for<2>([&](auto EZ) {
      constexpr int ey = decltype(EY)::value, ez = decltype(EZ)::value;
      constexpr int an = corner_id(AX, 1 - ey, 1 - ez);
      T t[3] = {T(0), T(0), T(0)};
      [[maybe_unused]] T tm[3] = {T(0), T(0), T(0)};
      static_for<2>([&](auto BY) {
        static_for<2>([&](auto BZ) {
          constexpr int by = decltype(BY)::value, bz = decltype(BZ)::value;
          constexpr int bn = corner_id(BX, by, bz);
          static_for<3>([&](auto C) {
            static_for<3>([&](auto C2) {
              constexpr int c = decltype(C)::value, c2 = decltype(C2)::value;
              constexpr int code = kKhatClass[(3 * an + c) * 24 + 3 * bn + c2];
              constexpr int cls = (code > 0 ? code : -code) - 1;
              const T k = code > 0 ? kv[cls] : -kv[cls];
              t[c] = fma(k, u[ey + by][ez + bz][c2], t[c]);
            });
            if constexpr (kMass) {
              constexpr int c = decltype(C)::value;
              constexpr int dist = (AX != BX) + ((1 - ey) != by) + ((1 - ez) != bz);
              tm[c] = fma(mv[dist], u[ey + by][ez + bz][c], tm[c]);
            }
          });
        });
      });
#pragma unroll
      for (int c = 0; c < 3; ++c) y[c] = fma(E[ey][ez], t[c], y[c]);
      if constexpr (kMass) {
        if (E[ey][ez] > T(0))
#pragma unroll
          for (int c = 0; c < 3; ++c) y[c] += tm[c];
      }
    });
  });
}

// Sweep the interior pencil (J, K) (padded coordinates, 1-based) for one
// realization lane, streaming x-planes: plane P feeds the output nodes P-1, P
// and P+1 through the element slabs with lower corner x = P-1 and x = P, so
// only the current plane (27 values), three partial outputs and two E slabs
// are live. Node P-1 is complete (and emitted) after plane P. Load(node, v3)
// produces the operator input at a node, Own(node, v3) runs once per node of
// the pencil with its input, Emit(node, own3, y3) receives the input and the
// operator output at the node.
template <class T, bool kMass = false, class Load, class Own, class Emit>
__device__ __forceinline__ void pencil_sweep(const Lattice& L, const typename KhatOf<T>::type& K, int J, int Kz,
                                             const T* __restrict__ E, Load load, Own own, Emit emit,
                                             const MassClasses<T>* M = nullptr) {
  const int Rp = L.Rp;
  T kv[kKhatClasses];  // class values in registers
#pragma unroll
  for (int i = 0; i < kKhatClasses; ++i) kv[i] = K.v[i];
  T mv[4] = {T(0), T(0), T(0), T(0)};
  if constexpr (kMass) {
#pragma unroll
    for (int i = 0; i < 4; ++i) mv[i] = M->v[i];
  }
  const size_t sxy = (size_t)L.NXp, sxz = (size_t)L.NXp * L.NYp;
  const size_t row0 = (size_t)(J + L.NYp * Kz) * L.NXp;  // padded node index of x = 0
  T ym[3] = {T(0), T(0), T(0)}, y0[3] = {T(0), T(0), T(0)}, yp[3];  // outputs at P-1, P, P+1
  T Eprev[2][2] = {{T(0), T(0)}, {T(0), T(0)}};                       // slab x = P-1 (x = 0: ghosts)
  T own_m[3] = {T(0), T(0), T(0)};                                     // input at node P-1
#pragma unroll 1
  for (int P = 1; P <= L.NX; ++P) {
    const size_t node = row0 + P;
    T pl[3][3][3];  // plane P: nodes (P, J-1+dy, K-1+dz)
#pragma unroll
    for (int dy = 0; dy < 3; ++dy)
#pragma unroll
      for (int dz = 0; dz < 3; ++dz) {
        load(node + (dy - 1) * sxy + (dz - 1) * sxz, pl[dy][dz]);
      }
    own(node, pl[1][1]);  // side effects at the plane's centre node (x = P)
    T Ecur[2][2];
#pragma unroll
    for (int ey = 0; ey < 2; ++ey)
#pragma unroll
      for (int ez = 0; ez < 2; ++ez) Ecur[ey][ez] = ldv(E + (node + (ey - 1) * sxy + (ez - 1) * sxz) * Rp);
#pragma unroll
    for (int c = 0; c < 3; ++c) yp[c] = T(0);
    slab_apply<T, 1, 0, kMass>(kv, pl, Ecur, yp, mv);   // slab P, output P+1
    slab_apply<T, 0, 0, kMass>(kv, pl, Ecur, y0, mv);   // slab P, output P
    slab_apply<T, 1, 1, kMass>(kv, pl, Eprev, y0, mv);  // slab P-1, output P
    slab_apply<T, 0, 1, kMass>(kv, pl, Eprev, ym, mv);  // slab P-1, output P-1
    if (P > 1) emit(node - 1, own_m, ym);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      ym[c] = y0[c];
      y0[c] = yp[c];
      own_m[c] = pl[1][1][c];
    }
#pragma unroll
    for (int ey = 0; ey < 2; ++ey)
#pragma unroll
      for (int ez = 0; ez < 2; ++ez) Eprev[ey][ez] = Ecur[ey][ez];
  }
  emit(row0 + L.NX, own_m, ym);  // the last node: plane NX+1 is a ghost plane
}

// Per-CTA reduction of per-realization partials over its warps (same lanes).
template <int NV>
__device__ __forceinline__ void cta_partial(const double (&v)[NV], double* __restrict__ out, int tile, int Rp, int rr) {
  __shared__ double sh[kWarps][NV][32];
  const int lane = threadIdx.x, w = threadIdx.y;
#pragma unroll
  for (int q = 0; q < NV; ++q) sh[w][q][lane] = v[q];
  __syncthreads();
  if (w == 0) {
#pragma unroll
    for (int q = 0; q < NV; ++q) {
      double s = 0;
#pragma unroll
      for (int ww = 0; ww < kWarps; ++ww) s += sh[ww][q][lane];
      out[((size_t)tile * Rp + rr) * NV + q] = s;
    }
  }
}

__device__ __forceinline__ void pencil_of(const Lattice& L, int& J, int& Kz, bool& valid) {
  const int tile = blockIdx.x;
  const int tj = tile % L.tiles_j, tk = tile / L.tiles_j;
  const int j = tj * kTJ + (threadIdx.y % kTJ), k = tk * kTK + (threadIdx.y / kTJ);
  valid = j < L.NY && k < L.NZ;
  J = j + 1;
  Kz = k + 1;
}

// ---------------------------------------------------------------- polynomial-chaos Galerkin product
// y_j = sum over the terms t of block j of c_t K(E_pos_t) u_k_t, FP64: the
// stochastic Galerkin matrix-vector product of PolynomialChaosSolverPCGMatrixCalculator.
// MultiplyWithMatrix (ISAAR.MSolve.Analyzers/PolynomialChaosSolverPCGMatrixCalculator.cs:1062-1089)
// on a structured lattice, each K_pos applied element by element from its
// field E_pos (value-class stencil, the pencil sweep of the FP64 residual).
// One thread per node pencil and output block (lane = block j); terms are
// accumulated in the reference's order (matrix, then input block) into the
// thread's own outputs.
__global__ void __launch_bounds__(128)
    k_pc_matvec(Lattice L, const __grid_constant__ KhatD K, const double* __restrict__ u,
                const double* __restrict__ Epc, int Mp, const uint8_t* __restrict__ mask,
                const int* __restrict__ term_ptr, const int* __restrict__ term_pos, const int* __restrict__ term_k,
                const double* __restrict__ term_c, int P, double* __restrict__ y) {
  int J, Kz;
  bool valid;
  pencil_of(L, J, Kz, valid);
  const int Pp = L.Rp;
  const int j = blockIdx.y * 32 + threadIdx.x;
  if (!valid || j >= P) return;
  Lattice LE = L;
  LE.Rp = Mp;  // the pencil sweep strides the element field by Rp
  for (int t = term_ptr[j]; t < term_ptr[j + 1]; ++t) {
    const int pos = term_pos[t], k = term_k[t];
    const double c = term_c[t];
    const bool first = t == term_ptr[j];
    auto load = [&](size_t node, double* o) {
#pragma unroll
      for (int cc = 0; cc < 3; ++cc) o[cc] = u[(node * 3 + cc) * Pp + k];
    };
    auto own = [](size_t, const double*) {};
    auto emit = [&](size_t node, const double*, const double* yy) {
      const uint32_t mk = mask[node];
#pragma unroll
      for (int cc = 0; cc < 3; ++cc) {
        const size_t o = (node * 3 + cc) * Pp + j;
        const double v = ((mk >> cc) & 1) ? 0.0 : c * yy[cc];
        y[o] = first ? v : y[o] + v;
      }
    };
    pencil_sweep<double>(LE, K, J, Kz, Epc + pos, load, own, emit);
  }
}

// E_pc[row(e)][0] = mean, E_pc[row(e)][1 + i] = mean * psi[i][e] (the field of
// the i-th expansion term, GaussianFileStochasticCoefficientsProvider
// GetCoefficientInternal scaled by the mean modulus)
__global__ void k_pc_fields(int ne, int m, int Mp, double mean, const double* __restrict__ psi,
                            const int* __restrict__ elem_row, double* __restrict__ Epc) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= ne) return;
  const size_t row = (size_t)elem_row[e];
  Epc[row * Mp] = mean;
  for (int i = 0; i < m; ++i) Epc[row * Mp + 1 + i] = mean * psi[(size_t)i * ne + e];
}

// block-major DOF vectors [P][n_dofs] <-> lattice layout [padded node][3][Pp]
__global__ void k_pc_scatter(int n_dofs, int P, int Pp, const int* __restrict__ rows, const double* __restrict__ in,
                             double* __restrict__ out) {
  const int d = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y;
  if (d < n_dofs && j < P) out[(size_t)rows[d] * Pp + j] = in[(size_t)j * n_dofs + d];
}
__global__ void k_pc_gather(int n_dofs, int P, int Pp, const int* __restrict__ rows, const double* __restrict__ in,
                            double* __restrict__ out) {
  const int d = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y;
  if (d < n_dofs && j < P) out[(size_t)j * n_dofs + d] = in[(size_t)rows[d] * Pp + j];
}

// ---------------------------------------------------------------- mbarrier and TMA helpers
// Every wait on an mbarrier is bounded: on expiry the kernel raises *err and
// stops streaming (the host reads the flag and returns MSG_ERR_TIMEOUT).
constexpr long kWaitLimit = 1L << 24;                    // try_wait polls before giving up

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
// Bounded wait for the phase with the given parity to complete.
__device__ __forceinline__ bool mbar_wait_n(uint64_t* bar, uint32_t parity, long limit) {
  const uint32_t a = smem_u32(bar);
  for (long i = 0; i < limit; ++i) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) { return mbar_wait_n(bar, parity, kWaitLimit); }

// Self-test of the bounded waits: one thread waits, with `polls` polls, on an
// mbarrier that nothing completes and records the expiry in *err, as every
// operator wait does; the kernel then returns normally.
__global__ void k_wait_selftest(long polls, int* err) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (threadIdx.x == 0 && !mbar_wait_n(&bar, 0, polls)) atomicExch(err, 1);
}
__device__ __forceinline__ void tma_load_5d(void* dst, const CUtensorMap* tm, int c0, int c1, int c2, int c3, int c4,
                                            uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.5d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5, %6}], "
      "[%7];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(tm)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* tm, int c0, int c1, int c2, int c3,
                                            uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
      "[%6];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(tm)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(bar))
      : "memory");
}

// ---------------------------------------------------------------- modal FP32 operator
// The element matrices of a cube are nearly diagonal in the element's Walsh
// modes. With the corner coordinates a = (ax, ay, az) in {0,1}^3 and the mode
// bits m = (mx, my, mz), s(a, m) = prod_d (2 a_d - 1)^{m_d} and T = s (x) I3
// (T T^T = 8 I), Km = T^T Khat T has 45 non-zeros in nine blocks (the rigid
// translations m = 0 are its null space):
//   V  {(1,x) (2,y) (4,z)}           [[a b b] [b a b] [b b a]]  (volumetric)
//   S  {(1,y) (2,x)} {(1,z) (4,x)} {(2,z) (4,y)}   [[a b] [b a]]  (linear shear)
//   P  {(3,x) (6,z)} {(3,y) (5,z)} {(5,x) (6,y)}   [[a b] [b a]]
//   T  {(3,z) (5,y) (6,x)}           [[a b b] [b a b] [b b a]]
//   D  (7,x) (7,y) (7,z)             a
// (mode m = mx + 2 my + 4 mz, component). The consistent mass is diagonal in
// the same modes. So Khat u = T (Km / 64) T^T u: the +-1 transforms factor
// per axis (sum and difference of two values), and the yz part of a plane
// is shared by the elements on both sides of it along x.
//
// A CTA owns a 3 x 3 tile of node pencils for 32 realizations and runs one
// warp per element pencil of the 4 x 4 that touch it (the tile's own
// elements plus one halo row and column below; the 7 halo pencils are also
// computed by the neighbouring CTA). Per x-plane P every element warp turns
// its 4 plane nodes into 4 yz-modes per component, combines them with the
// previous plane's modes into the element's 24 modes, applies the blocks,
// and folds the result back onto the yz-modes of planes P-1 and P; the P-1
// part completes that plane and goes back to its 4 corner nodes. The corner
// contributions meet in a shared-memory exchange buffer, where the warp that
// owns node pencil (J, K) sums the four elements around it in fixed order,
// so results stay deterministic. About 150 FP32 operations per element and
// plane instead of the 576 FMAs of a dense Khat row block per node. The
// output is not masked here: constrained components of p are zero, so p.q
// is unaffected, and k_update leaves the constrained components of r at zero.
//
// The kernel is persistent (one CTA per SM walks work items, a tile and a
// realization group each), with a dedicated TMA producer warp filling the
// same 4-stage mbarrier ring as the dense operator, and an mbarrier (bounded
// waits, like every other wait here) in place of a CTA barrier between the
// element and node phases of a plane.
template <class T> struct ModalCT {
  T vd, vb;  // V: a - b, b
  T sa, sb;  // S: a, b
  T pa, pb;  // P: a, b
  T td, tb;  // T: a - b, b
  T da;      // D
  T m[8];    // mass per mode (0 when no mass term)
};
using ModalC = ModalCT<float>;
using ModalCD = ModalCT<double>;

template <class T> __device__ __forceinline__ T fmx(T a, T b, T c);
template <> __device__ __forceinline__ float fmx<float>(float a, float b, float c) { return fmaf(a, b, c); }
template <> __device__ __forceinline__ double fmx<double>(double a, double b, double c) { return fma(a, b, c); }
// Two realizations in one register pair: Blackwell's packed FP32 instructions
// (one issue slot for both halves of a float2)
__device__ __forceinline__ float2 operator+(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 operator-(float2 a, float2 b) { return __ffma2_rn(b, make_float2(-1.f, -1.f), a); }
__device__ __forceinline__ float2 operator*(float2 a, float2 b) { return __fmul2_rn(a, b); }
template <> __device__ __forceinline__ float2 fmx<float2>(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
template <class T> __device__ __forceinline__ T zero_of() { return T(0); }
template <> __device__ __forceinline__ float2 zero_of<float2>() { return make_float2(0.f, 0.f); }

constexpr int kMJ = 3, kMK = 3;                       // node pencils per tile
constexpr int kMEJ = kMJ + 1, kMEK = kMK + 1;         // element pencils per tile
constexpr int kMWarps = kMEJ * kMEK;                  // 16 element warps (+ 1 producer: 96 registers a thread)
constexpr int kMPJ = kMJ + 2, kMPK = kMK + 2;         // node patch per plane
constexpr int kMPlaneFloats = 32 * 3 * kMPJ * kMPK;   // r, q or p patch of a plane: 2400
constexpr int kMNodeFloats = 32 * kMPJ * kMPK;        // dinv patch: 800
constexpr int kMEFloats = 32 * kMEJ * kMEK;           // E patch: 512
constexpr int kMDFloats = 32 * 3 * kMJ * kMK;         // d of the tile's own nodes: 864
// stage: r | q | p | dinv | E | d (each patch a multiple of 128 bytes)
constexpr int kMOffR = 0, kMOffQ = kMPlaneFloats, kMOffP = 2 * kMPlaneFloats, kMOffDinv = 3 * kMPlaneFloats;
constexpr int kMOffE = kMOffDinv + kMNodeFloats, kMOffD = kMOffE + kMEFloats;
constexpr int kMStageFloats = kMOffD + kMDFloats;     // 9,376 floats, 37,504 bytes
constexpr uint32_t kMStageBytes = kMStageFloats * 4;
constexpr int kMStages = 3;
constexpr int kMXFloats = kMWarps * 4 * 3 * 32;       // exchange buffer: element x corner x component x lane
constexpr int kMThreads = 32 * (kMWarps + 1);         // + 1 TMA producer warp
constexpr size_t kMSmem = 128 + sizeof(float) * ((size_t)kMStages * kMStageFloats + 2 * (size_t)kMXFloats) +
                          sizeof(double) * 4 * kMJ * kMK * 32 + sizeof(uint64_t) * (2 * kMStages);
static_assert(kMSmem <= 227 * 1024, "modal operator shared memory");

// yz transform of one plane's 4 nodes u[ay][az] into the modes B[my + 2 mz]
template <class T>
__device__ __forceinline__ void yz_forward(const T (&u)[2][2][3], T (&B)[3][4]) {
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const T z00 = u[0][0][c] + u[0][1][c], z01 = u[0][1][c] - u[0][0][c];
    const T z10 = u[1][0][c] + u[1][1][c], z11 = u[1][1][c] - u[1][0][c];
    B[c][0] = z00 + z10;
    B[c][1] = z10 - z00;
    B[c][2] = z01 + z11;
    B[c][3] = z11 - z01;
  }
}

// inverse of yz_forward up to the factor 4 (the transpose of the same signs)
template <class T>
__device__ __forceinline__ void yz_inverse(const T (&B)[3][4], T (&y)[2][2][3]) {
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const T a00 = B[c][0] - B[c][1], a10 = B[c][0] + B[c][1];
    const T a01 = B[c][2] - B[c][3], a11 = B[c][2] + B[c][3];
    y[0][0][c] = a00 - a01;
    y[0][1][c] = a00 + a01;
    y[1][0][c] = a10 - a11;
    y[1][1][c] = a10 + a11;
  }
}

// One element between planes P-1 (yz-modes Bp) and P (Bc): T0 += the part of
// E Km/64 u (+ mass) that lands on plane P-1, C1 = the part on plane P, both
// in yz-modes. y0 / y1 hold the element modes with mx = 0 / 1, as [c][my + 2 mz].
template <bool kMass, class T>
__device__ __forceinline__ void modal_apply(const ModalCT<T>& C, T E, const T (&Bp)[3][4], const T (&Bc)[3][4],
                                            T (&T0)[3][4], T (&C1)[3][4]) {
  T y0[3][4], y1[3][4];
  auto U0 = [&](int q, int c) { return Bc[c][q] + Bp[c][q]; };
  auto U1 = [&](int q, int c) { return Bc[c][q] - Bp[c][q]; };
  const T Evd = E * C.vd, Evb = E * C.vb, Esa = E * C.sa, Esb = E * C.sb;
  const T Epa = E * C.pa, Epb = E * C.pb, Etd = E * C.td, Etb = E * C.tb, Eda = E * C.da;
  {  // V
    const T a = U1(0, 0), b = U0(1, 1), c = U0(2, 2);
    const T t = Evb * (a + b + c);
    y1[0][0] = fmx(Evd, a, t);
    y0[1][1] = fmx(Evd, b, t);
    y0[2][2] = fmx(Evd, c, t);
  }
  {  // S
    T a = U1(0, 1), b = U0(1, 0);
    y1[1][0] = fmx(Esa, a, Esb * b);
    y0[0][1] = fmx(Esa, b, Esb * a);
    a = U1(0, 2), b = U0(2, 0);
    y1[2][0] = fmx(Esa, a, Esb * b);
    y0[0][2] = fmx(Esa, b, Esb * a);
    a = U0(1, 2), b = U0(2, 1);
    y0[2][1] = fmx(Esa, a, Esb * b);
    y0[1][2] = fmx(Esa, b, Esb * a);
  }
  {  // P
    T a = U1(1, 0), b = U0(3, 2);
    y1[0][1] = fmx(Epa, a, Epb * b);
    y0[2][3] = fmx(Epa, b, Epb * a);
    a = U1(1, 1), b = U1(2, 2);
    y1[1][1] = fmx(Epa, a, Epb * b);
    y1[2][2] = fmx(Epa, b, Epb * a);
    a = U1(2, 0), b = U0(3, 1);
    y1[0][2] = fmx(Epa, a, Epb * b);
    y0[1][3] = fmx(Epa, b, Epb * a);
  }
  {  // T
    const T a = U1(1, 2), b = U1(2, 1), c = U0(3, 0);
    const T t = Etb * (a + b + c);
    y1[2][1] = fmx(Etd, a, t);
    y1[1][2] = fmx(Etd, b, t);
    y0[0][3] = fmx(Etd, c, t);
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) {  // D and the null modes
    y1[c][3] = Eda * U1(3, c);
    y0[c][0] = zero_of<T>();
  }
  if constexpr (kMass) {
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        y0[c][q] = fmx(C.m[2 * q], U0(q, c), y0[c][q]);
        y1[c][q] = fmx(C.m[2 * q + 1], U1(q, c), y1[c][q]);
      }
  }
#pragma unroll
  for (int q = 0; q < 4; ++q)
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      T0[c][q] = (T0[c][q] + y0[c][q]) - y1[c][q];
      C1[c][q] = y0[c][q] + y1[c][q];
    }
}

// One whole inner PCG iteration per launch (single-reduction form). Launch k+1
// receives r_k, q_k = K p_k, p_k, alpha_k and beta_{k+1} and, at every node,
//   r_{k+1} = r_k - alpha_k q_k,  p_{k+1} = dinv r_{k+1} + beta_{k+1} p_k,
//   d += alpha_k p_k (the FP32 solution correction),
// then q_{k+1} = K p_{k+1} (masked) with the partials p.q, (dinv r).q,
// q.dinv.q and (dinv r).r of p_{k+1}, r_{k+1}, q_{k+1}. The scalar kernel that
// follows forms alpha_{k+1} = gamma_{k+1} / p.q from the gamma of r_{k+1}
// itself and the next gamma by the expansion of (dinv r_{k+2}).r_{k+2},
//   gamma_{k+2} = gamma_{k+1} - 2 alpha (dinv r).q + alpha^2 q.dinv.q,
// so r never needs a pass of its own (and the expansion never runs for more
// than one step, which keeps the FP32 iteration count of the two-pass loop). Each stage carries the plane's r, q, p and dinv patches with halo (and
// the tile's d); the element warps form p_{k+1} at their corners on the fly,
// and the owner of a node pencil writes r, p and d back. r, q and p each have
// a second buffer: neighbouring CTAs still read the old values in their halos.
constexpr int kMParts = 4;  // partials per realization and tile: p.q, (dinv r).q, q.dinv.q, (dinv r).r
template <bool kMass>
__global__ void __launch_bounds__(kMThreads, 1)
    k_op_modal(Lattice L, const __grid_constant__ ModalC C, const __grid_constant__ CUtensorMap tm_r,
               const __grid_constant__ CUtensorMap tm_q, const __grid_constant__ CUtensorMap tm_p,
               const __grid_constant__ CUtensorMap tm_dinv, const __grid_constant__ CUtensorMap tm_e,
               const __grid_constant__ CUtensorMap tm_d, int tiles_j, int n_tiles, int n_items,
               const uint8_t* __restrict__ mask, const float* __restrict__ alpha, const float* __restrict__ beta,
               float* __restrict__ r_out, float* __restrict__ p_out, float* __restrict__ q_out, float* __restrict__ d,
               double* __restrict__ partial, int* __restrict__ err) {
  extern __shared__ __align__(128) float smem_dyn[];
  float* smem = smem_dyn + (((128u - (smem_u32(smem_dyn) & 127u)) & 127u) >> 2);
  float* xbuf = smem + kMStages * kMStageFloats;                            // 2 exchange buffers
  double* red = reinterpret_cast<double*>(xbuf + 2 * kMXFloats);            // [parts][node pencils][32]
  uint64_t* full = reinterpret_cast<uint64_t*>(red + kMParts * kMJ * kMK * 32);
  uint64_t* empty = full + kMStages;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int NX = L.NX, Rp = L.Rp;
  if (threadIdx.x == 0) {
    for (int st = 0; st < kMStages; ++st) {
      mbar_init(&full[st], 1);
      mbar_init(&empty[st], kMWarps);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (w == kMWarps) {
    // producer: plane P of every work item, in the consumers' order
    if (lane == 0) {
      uint32_t seq = 0;
      for (int item = blockIdx.x; item < n_items; item += gridDim.x) {
        const int tile = item % n_tiles, g32 = (item / n_tiles) * 32;
        const int J0 = 1 + (tile % tiles_j) * kMJ, K0 = 1 + (tile / tiles_j) * kMK;
        for (int P = 1; P <= NX; ++P, ++seq) {
          const int st = seq % kMStages;
          const uint32_t use = seq / kMStages;
          if (use > 0 && !mbar_wait(&empty[st], (use - 1) & 1)) {
            atomicExch(err, 1);
            return;
          }
          float* dst = smem + st * kMStageFloats;
          mbar_expect_tx(&full[st], kMStageBytes);
          tma_load_5d(dst + kMOffR, &tm_r, g32, 0, P, J0 - 1, K0 - 1, &full[st]);
          tma_load_5d(dst + kMOffQ, &tm_q, g32, 0, P, J0 - 1, K0 - 1, &full[st]);
          tma_load_5d(dst + kMOffP, &tm_p, g32, 0, P, J0 - 1, K0 - 1, &full[st]);
          tma_load_4d(dst + kMOffDinv, &tm_dinv, g32, P, J0 - 1, K0 - 1, &full[st]);
          tma_load_4d(dst + kMOffE, &tm_e, g32, P - 1, J0 - 1, K0 - 1, &full[st]);
          tma_load_5d(dst + kMOffD, &tm_d, g32, 0, P, J0, K0, &full[st]);
        }
      }
    }
    return;
  }
  const int ej = w % kMEJ, ek = w / kMEJ;
  const bool node_warp = ej >= 1 && ek >= 1;
  uint32_t seq = 0;
  int xsel = 0;
  bool dead = false;  // a stage never arrived: finish the walk without data (err is set)
  // barrier of the consumer warps between the element and the node phase of a
  // plane; every consumer warp passes the same sequence of them, error or not
  auto csync = [&]() { asm volatile("bar.sync 1, %0;" ::"r"(kMWarps * 32) : "memory"); };
  for (int item = blockIdx.x; item < n_items; item += gridDim.x) {
    const int tile = item % n_tiles, g32 = (item / n_tiles) * 32;
    const int J0 = 1 + (tile % tiles_j) * kMJ, K0 = 1 + (tile / tiles_j) * kMK;
    const int Je = J0 - 1 + ej, Ke = K0 - 1 + ek;  // element pencil (lower corner), padded
    // real elements have lower corners 1..NY-1 (1..NZ-1); others are ghosts
    auto realj = [&](int j) { return j >= 1 && j <= L.NY - 1; };
    auto realk = [&](int k) { return k >= 1 && k <= L.NZ - 1; };
    const bool real = realj(Je) && realk(Ke);
    const bool node_ok = node_warp && Je <= L.NY && Ke <= L.NZ;
    const bool r00 = real, r10 = realj(Je - 1) && realk(Ke);
    const bool r01 = realj(Je) && realk(Ke - 1), r11 = realj(Je - 1) && realk(Ke - 1);
    const size_t nrow = ((size_t)Je + (size_t)L.NYp * Ke) * L.NXp;  // padded node (0, Je, Ke)
    const int rr = g32 + lane;
    const float al = alpha[rr], be = beta[rr];
    float Bp[3][4], T0[3][4];
    float op[3] = {0.f, 0.f, 0.f}, orr[3] = {0.f, 0.f, 0.f}, odv = 0.f;  // p, r, dinv at the own node
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int qq = 0; qq < 4; ++qq) T0[c][qq] = 0.f;
    double acc_pq = 0.0, acc_zq = 0.0, acc_qq = 0.0, acc_zr = 0.0;
    uint32_t mreg = 0;  // constraint bits of plane base + lane of the own pencil
    // node phase of plane X: sum the corner contributions of the 4 elements
    auto node_phase = [&](int X) {
      if (((X - 1) & 31) == 0) {
        const int pl = X + lane;
        mreg = (pl <= NX) ? mask[nrow + pl] : 0u;
      }
      const uint32_t mk = __shfl_sync(0xffffffffu, mreg, (X - 1) & 31);
      const float* xb = xbuf + xsel * kMXFloats;
      const size_t node = nrow + X;
      // products in FP64: a fast-converging realization drives r and q towards the
      // bottom of the FP32 range, where FP32 squares would underflow
      double spq = 0.0, szq = 0.0, sqq = 0.0, szr = 0.0;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        float y = 0.f;
        if (r00) y += xb[((w * 4 + 0) * 3 + c) * 32 + lane];
        if (r10) y += xb[(((w - 1) * 4 + 1) * 3 + c) * 32 + lane];
        if (r01) y += xb[(((w - kMEJ) * 4 + 2) * 3 + c) * 32 + lane];
        if (r11) y += xb[(((w - kMEJ - 1) * 4 + 3) * 3 + c) * 32 + lane];
        y = ((mk >> c) & 1) ? 0.f : y;
        q_out[(node * 3 + c) * Rp + rr] = y;
        const double yd = (double)y, rd = (double)orr[c];
        spq = fma((double)op[c], yd, spq);
        szq = fma(rd, yd, szq);
        sqq = fma(yd, yd, sqq);
        szr = fma(rd, rd, szr);
      }
      const double dvd = (double)odv;
      acc_pq += spq;
      acc_zq += dvd * szq;
      acc_qq += dvd * sqq;
      acc_zr += dvd * szr;
    };
    auto emit_corners = [&](const float (&B)[3][4]) {
      float y[2][2][3];
      yz_inverse(B, y);
      float* xb = xbuf + xsel * kMXFloats;
#pragma unroll
      for (int ay = 0; ay < 2; ++ay)
#pragma unroll
        for (int az = 0; az < 2; ++az)
#pragma unroll
          for (int c = 0; c < 3; ++c) xb[((w * 4 + ay + 2 * az) * 3 + c) * 32 + lane] = y[ay][az][c];
    };
    for (int P = 1; P <= NX; ++P, ++seq) {
      const int st = seq % kMStages;
      if (!dead && !mbar_wait(&full[st], (seq / kMStages) & 1)) {
        atomicExch(err, 1);
        dead = true;
      }
      const float* pt = smem + st * kMStageFloats;
      // p_{k+1} at the element's 4 plane corners: dinv (r - alpha q) + beta p_k
      float u[2][2][3], rc[3], dvc = 0.f;
#pragma unroll
      for (int ay = 0; ay < 2; ++ay)
#pragma unroll
        for (int az = 0; az < 2; ++az) {
          const int o = (ek + az) * kMPJ + (ej + ay);
          const float dv = pt[kMOffDinv + o * 32 + lane];
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            const int i = (o * 3 + c) * 32 + lane;
            const float rn = fmaf(-al, pt[kMOffQ + i], pt[kMOffR + i]);
            u[ay][az][c] = fmaf(dv, rn, be * pt[kMOffP + i]);
            if (ay == 0 && az == 0) rc[c] = rn;
          }
          if (ay == 0 && az == 0) dvc = dv;
        }
      const float E = pt[kMOffE + w * 32 + lane];  // element (P-1, Je, Ke)
      if (node_ok) {
        // the owner writes r_{k+1}, p_{k+1} and d += alpha_k p_k of node (P, Je, Ke)
        const int o = ek * kMPJ + ej, od = (ek - 1) * kMJ + (ej - 1);
        const size_t node = nrow + P;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const float pold = pt[kMOffP + (o * 3 + c) * 32 + lane];
          const float dn = fmaf(al, pold, pt[kMOffD + (od * 3 + c) * 32 + lane]);
          r_out[(node * 3 + c) * Rp + rr] = rc[c];
          p_out[(node * 3 + c) * Rp + rr] = u[0][0][c];
          d[(node * 3 + c) * Rp + rr] = dn;
        }
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(&empty[st]);
      float Bc[3][4];
      yz_forward(u, Bc);
      if (P >= 2) {
        if (real) {
          float C1[3][4];
          modal_apply<kMass>(C, E, Bp, Bc, T0, C1);
          emit_corners(T0);
#pragma unroll
          for (int c = 0; c < 3; ++c)
#pragma unroll
            for (int qq = 0; qq < 4; ++qq) T0[c][qq] = C1[c][qq];
        }
        csync();
        if (node_ok) node_phase(P - 1);
        xsel ^= 1;
      }
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        op[c] = u[0][0][c];
        orr[c] = rc[c];
        odv = dvc;
#pragma unroll
        for (int qq = 0; qq < 4; ++qq) Bp[c][qq] = Bc[c][qq];
      }
    }
    // plane NX: the slab above it is a ghost, so the pending part is complete
    if (real) emit_corners(T0);
    csync();
    if (node_ok) node_phase(NX);
    xsel ^= 1;
    if (node_warp) {
      const int nw = (ek - 1) * kMJ + (ej - 1);
      red[(0 * kMJ * kMK + nw) * 32 + lane] = acc_pq;
      red[(1 * kMJ * kMK + nw) * 32 + lane] = acc_zq;
      red[(2 * kMJ * kMK + nw) * 32 + lane] = acc_qq;
      red[(3 * kMJ * kMK + nw) * 32 + lane] = acc_zr;
    }
    csync();
    if (w < kMParts) {
      double sum = 0.0;
#pragma unroll
      for (int i = 0; i < kMJ * kMK; ++i) sum += red[(w * kMJ * kMK + i) * 32 + lane];
      partial[((size_t)tile * Rp + rr) * kMParts + w] = sum;
    }
  }
}

// ---------------------------------------------------------------- multigrid level operator
// The Walsh-mode operator of one lattice level (same tiling, TMA ring,
// exchange buffer and bounded waits as k_op_modal), with the node phase of one
// step of the multigrid-preconditioned loop:
//   kLvlStart : level 0, first step of an iteration. Corner input
//               x0 = omega dinv (r - alpha q) (the first Jacobi sweep from zero
//               on the updated residual); the owner writes r' = r - alpha q
//               (out2) and x0 (out3); out = r' - A x0; partial r'.r'.
//   kLvlResid : out = b - A u.
//   kLvlSmooth: out = u + omega dinv (b - A u) (damped Jacobi sweep); partial
//               out.b when partial is given.
//   kLvlPcgZ  : level 0, search direction. Corner input p = z + beta p_old;
//               the owner writes p (out2) and d += alpha p_old; out = A p;
//               partial p.(A p).
// Every output is masked (constrained components 0). Per-realization partials
// are summed in a fixed order (node pencil, then plane), so they do not depend
// on the batch.
enum { kLvlStart = 0, kLvlResid = 1, kLvlSmooth = 2, kLvlPcgZ = 3 };
template <int kMode> struct LvlStage {
  static constexpr bool kTwo = kMode == kLvlStart || kMode == kLvlPcgZ;  // two vector patches
  static constexpr int kOffA = 0;              // r (start), z (direction) or u
  static constexpr int kOffB = kMPlaneFloats;  // q (start) or p_old (direction)
  static constexpr int kOffN = (kTwo ? 2 : 1) * kMPlaneFloats;                 // dinv patch (start)
  static constexpr int kOffE = kOffN + (kMode == kLvlStart ? kMNodeFloats : 0);
  static constexpr int kOffD = kOffE + kMEFloats;                              // d of the tile (direction)
  static constexpr int kFloats = kOffD + (kMode == kLvlPcgZ ? kMDFloats : 0);
  static constexpr uint32_t kBytes = kFloats * 4;
  static constexpr size_t kSmem = 128 + sizeof(float) * ((size_t)kMStages * kFloats + 2 * (size_t)kMXFloats) +
                                  sizeof(double) * kMJ * kMK * 32 + sizeof(uint64_t) * (2 * kMStages);
};
static_assert(LvlStage<kLvlResid>::kOffB == kMPlaneFloats && LvlStage<kLvlSmooth>::kOffB == kMPlaneFloats,
              "the second vector patch follows the first");
static_assert(LvlStage<kLvlStart>::kBytes % 128 == 0 && LvlStage<kLvlResid>::kBytes % 128 == 0 &&
                  LvlStage<kLvlPcgZ>::kBytes % 128 == 0,
              "stage alignment");
static_assert(LvlStage<kLvlPcgZ>::kSmem <= 227 * 1024 && LvlStage<kLvlStart>::kSmem <= 227 * 1024, "level smem");

template <int kMode, bool kMass>
__global__ void __launch_bounds__(kMThreads, 1)
    k_lvl_op(Lattice L, const __grid_constant__ ModalC C, const __grid_constant__ CUtensorMap tm_a,
             const __grid_constant__ CUtensorMap tm_b, const __grid_constant__ CUtensorMap tm_n,
             const __grid_constant__ CUtensorMap tm_e, const __grid_constant__ CUtensorMap tm_d, int tiles_j,
             int n_tiles, int n_items, const uint8_t* __restrict__ mask, const float* __restrict__ b,
             const float* __restrict__ dinv, float omega, const float* __restrict__ alpha,
             const float* __restrict__ beta, float* __restrict__ out, float* __restrict__ out2,
             float* __restrict__ out3, float* __restrict__ d, double* __restrict__ partial, int pstride,
             int* __restrict__ err) {
  using S = LvlStage<kMode>;
  extern __shared__ __align__(128) float smem_dyn[];
  float* smem = smem_dyn + (((128u - (smem_u32(smem_dyn) & 127u)) & 127u) >> 2);
  float* xbuf = smem + kMStages * S::kFloats;
  double* red = reinterpret_cast<double*>(xbuf + 2 * kMXFloats);  // [node pencils][32]
  uint64_t* full = reinterpret_cast<uint64_t*>(red + kMJ * kMK * 32);
  uint64_t* empty = full + kMStages;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int NX = L.NX, Rp = L.Rp;
  if (threadIdx.x == 0) {
    for (int st = 0; st < kMStages; ++st) {
      mbar_init(&full[st], 1);
      mbar_init(&empty[st], kMWarps);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (w == kMWarps) {
    if (lane == 0) {
      uint32_t seq = 0;
      for (int item = blockIdx.x; item < n_items; item += gridDim.x) {
        const int tile = item % n_tiles, g32 = (item / n_tiles) * 32;
        const int J0 = 1 + (tile % tiles_j) * kMJ, K0 = 1 + (tile / tiles_j) * kMK;
        for (int P = 1; P <= NX; ++P, ++seq) {
          const int st = seq % kMStages;
          const uint32_t use = seq / kMStages;
          if (use > 0 && !mbar_wait(&empty[st], (use - 1) & 1)) {
            atomicExch(err, 1);
            return;
          }
          float* dst = smem + st * S::kFloats;
          mbar_expect_tx(&full[st], S::kBytes);
          tma_load_5d(dst + S::kOffA, &tm_a, g32, 0, P, J0 - 1, K0 - 1, &full[st]);
          if constexpr (S::kTwo) tma_load_5d(dst + S::kOffB, &tm_b, g32, 0, P, J0 - 1, K0 - 1, &full[st]);
          if constexpr (kMode == kLvlStart) tma_load_4d(dst + S::kOffN, &tm_n, g32, P, J0 - 1, K0 - 1, &full[st]);
          tma_load_4d(dst + S::kOffE, &tm_e, g32, P - 1, J0 - 1, K0 - 1, &full[st]);
          if constexpr (kMode == kLvlPcgZ) tma_load_5d(dst + S::kOffD, &tm_d, g32, 0, P, J0, K0, &full[st]);
        }
      }
    }
    return;
  }
  const int ej = w % kMEJ, ek = w / kMEJ;
  const bool node_warp = ej >= 1 && ek >= 1;
  uint32_t seq = 0;
  int xsel = 0;
  bool dead = false;
  auto csync = [&]() { asm volatile("bar.sync 1, %0;" ::"r"(kMWarps * 32) : "memory"); };
  for (int item = blockIdx.x; item < n_items; item += gridDim.x) {
    const int tile = item % n_tiles, g32 = (item / n_tiles) * 32;
    const int J0 = 1 + (tile % tiles_j) * kMJ, K0 = 1 + (tile / tiles_j) * kMK;
    const int Je = J0 - 1 + ej, Ke = K0 - 1 + ek;
    auto realj = [&](int j) { return j >= 1 && j <= L.NY - 1; };
    auto realk = [&](int k) { return k >= 1 && k <= L.NZ - 1; };
    const bool real = realj(Je) && realk(Ke);
    const bool node_ok = node_warp && Je <= L.NY && Ke <= L.NZ;
    const bool r00 = real, r10 = realj(Je - 1) && realk(Ke);
    const bool r01 = realj(Je) && realk(Ke - 1), r11 = realj(Je - 1) && realk(Ke - 1);
    const size_t nrow = ((size_t)Je + (size_t)L.NYp * Ke) * L.NXp;
    const int rr = g32 + lane;
    float al = 0.f, be = 0.f;
    if constexpr (kMode == kLvlStart || kMode == kLvlPcgZ) al = alpha[rr];
    if constexpr (kMode == kLvlPcgZ) be = beta[rr];
    float Bp[3][4], T0[3][4];
    float ou[3] = {0.f, 0.f, 0.f}, orc[3] = {0.f, 0.f, 0.f};  // corner input and r' at the own node, last plane
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int qq = 0; qq < 4; ++qq) T0[c][qq] = 0.f;
    double acc = 0.0;
    uint32_t mreg = 0;
    auto node_phase = [&](int X) {
      if (((X - 1) & 31) == 0) {
        const int pl = X + lane;
        mreg = (pl <= NX) ? mask[nrow + pl] : 0u;
      }
      const uint32_t mk = __shfl_sync(0xffffffffu, mreg, (X - 1) & 31);
      const float* xb = xbuf + xsel * kMXFloats;
      const size_t node = nrow + X;
      float wdv = 0.f;
      if constexpr (kMode == kLvlSmooth) wdv = omega * dinv[node * Rp + rr];
      double sacc = 0.0;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        float y = 0.f;
        if (r00) y += xb[((w * 4 + 0) * 3 + c) * 32 + lane];
        if (r10) y += xb[(((w - 1) * 4 + 1) * 3 + c) * 32 + lane];
        if (r01) y += xb[(((w - kMEJ) * 4 + 2) * 3 + c) * 32 + lane];
        if (r11) y += xb[(((w - kMEJ - 1) * 4 + 3) * 3 + c) * 32 + lane];
        const size_t o = (node * 3 + c) * Rp + rr;
        const bool fixed = (mk >> c) & 1;
        float v;
        if constexpr (kMode == kLvlStart) {
          v = fixed ? 0.f : orc[c] - y;
          sacc = fma((double)orc[c], (double)orc[c], sacc);
        } else if constexpr (kMode == kLvlResid) {
          v = fixed ? 0.f : b[o] - y;
        } else if constexpr (kMode == kLvlSmooth) {
          const float bv = b[o];
          v = fixed ? 0.f : fmaf(wdv, bv - y, ou[c]);
          sacc = fma((double)v, (double)bv, sacc);
        } else {
          v = fixed ? 0.f : y;
          sacc = fma((double)ou[c], (double)v, sacc);
        }
        out[o] = v;
      }
      acc += sacc;
    };
    auto emit_corners = [&](const float (&B)[3][4]) {
      float y[2][2][3];
      yz_inverse(B, y);
      float* xb = xbuf + xsel * kMXFloats;
#pragma unroll
      for (int ay = 0; ay < 2; ++ay)
#pragma unroll
        for (int az = 0; az < 2; ++az)
#pragma unroll
          for (int c = 0; c < 3; ++c) xb[((w * 4 + ay + 2 * az) * 3 + c) * 32 + lane] = y[ay][az][c];
    };
    for (int P = 1; P <= NX; ++P, ++seq) {
      const int st = seq % kMStages;
      if (!dead && !mbar_wait(&full[st], (seq / kMStages) & 1)) {
        atomicExch(err, 1);
        dead = true;
      }
      const float* pt = smem + st * S::kFloats;
      float u[2][2][3], rc[3] = {0.f, 0.f, 0.f};
#pragma unroll
      for (int ay = 0; ay < 2; ++ay)
#pragma unroll
        for (int az = 0; az < 2; ++az) {
          const int o = (ek + az) * kMPJ + (ej + ay);
          float wdv = 0.f;
          if constexpr (kMode == kLvlStart) wdv = omega * pt[S::kOffN + o * 32 + lane];
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            const int i = (o * 3 + c) * 32 + lane;
            if constexpr (kMode == kLvlStart) {
              const float rn = fmaf(-al, pt[S::kOffB + i], pt[S::kOffA + i]);
              u[ay][az][c] = wdv * rn;
              if (ay == 0 && az == 0) rc[c] = rn;
            } else if constexpr (kMode == kLvlPcgZ) {
              u[ay][az][c] = fmaf(be, pt[S::kOffB + i], pt[S::kOffA + i]);
            } else {
              u[ay][az][c] = pt[S::kOffA + i];
            }
          }
        }
      const float E = pt[S::kOffE + w * 32 + lane];
      if constexpr (kMode == kLvlStart || kMode == kLvlPcgZ) {
        if (node_ok) {
          const size_t node = nrow + P;
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            const size_t o = (node * 3 + c) * Rp + rr;
            if constexpr (kMode == kLvlStart) {
              out2[o] = rc[c];
              if (out3 != nullptr) out3[o] = u[0][0][c];
            } else {
              const int op = ek * kMPJ + ej, od = (ek - 1) * kMJ + (ej - 1);
              const float pold = pt[S::kOffB + (op * 3 + c) * 32 + lane];
              out2[o] = u[0][0][c];
              d[o] = fmaf(al, pold, pt[S::kOffD + (od * 3 + c) * 32 + lane]);
            }
          }
        }
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(&empty[st]);
      float Bc[3][4];
      yz_forward(u, Bc);
      if (P >= 2) {
        if (real) {
          float C1[3][4];
          modal_apply<kMass>(C, E, Bp, Bc, T0, C1);
          emit_corners(T0);
#pragma unroll
          for (int c = 0; c < 3; ++c)
#pragma unroll
            for (int qq = 0; qq < 4; ++qq) T0[c][qq] = C1[c][qq];
        }
        csync();
        if (node_ok) node_phase(P - 1);
        xsel ^= 1;
      }
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        ou[c] = u[0][0][c];
        orc[c] = rc[c];
#pragma unroll
        for (int qq = 0; qq < 4; ++qq) Bp[c][qq] = Bc[c][qq];
      }
    }
    if (real) emit_corners(T0);
    csync();
    if (node_ok) node_phase(NX);
    xsel ^= 1;
    if (kMode != kLvlResid && partial != nullptr) {
      if (node_warp) red[((ek - 1) * kMJ + (ej - 1)) * 32 + lane] = acc;
      csync();
      if (w == 0) {
        double sum = 0.0;
#pragma unroll
        for (int i = 0; i < kMJ * kMK; ++i) sum += red[i * 32 + lane];
        partial[((size_t)tile * Rp + rr) * pstride] = sum;
      }
    }
  }
}

// ---------------------------------------------------------------- tensor-core element product (level 0)
// k_lvl_tc<kLvlPcgZ>: the level-0 search-direction launch of the multigrid
// loop, with k_lvl_op<kLvlPcgZ>'s inputs, outputs, tiling and node phase, but
// the element product on the 5th-generation tensor cores (tcgen05.mma,
// kind::tf32, accumulators in tensor memory) instead of the Walsh modes. For
// the element pencils of an x-slab,
//   y_e = E_e (cK Khat) u_e
// is a product D[(element, realization)][output DOF] = sum over four corner
// pairs of U_pair [128 x 8] B_pair^T [8 x N]: a corner pair (ax, ay) covers the
// two corners az = 0, 1 of the element (slots 0-2 and 3-5 of an 8-slot K
// group; slots 6-7 are zero), so one node-pair group of a plane serves the
// element pencils on both of its sides. An M = 128 tile is the 4 element
// pencils along y of one z row, 32 realizations each; it reads 4 consecutive
// 1 KB groups (K-major core matrices of 8 realizations x 4 slots, no swizzle:
// a realization's 8 slots are two 16-byte rows, LBO 128 B between the slot
// halves, SBO 256 B between 8-realization groups). TF32 with a three-term
// split keeps FP32-level accuracy:
//   U = U_hi + U_lo (U_hi: U with the low 13 mantissa bits cleared),
//   cK Khat = B_hi + B_lo,  U Khat ~ U_hi [B_hi | B_lo] (N = 64) + U_lo B_hi (N = 32).
// Output column n = ((ax' 2 + ay') 2 + az') 3 + c'; columns 0-11 land on plane
// P-1, 12-23 on plane P (carried to the next slab, as the Walsh kernels carry
// C1). Per plane: every element warp forms p = z + beta p_old at the two
// nodes of its node-pair group (y = ej, z = ek; the last element column also
// the group at y = 4), splits it and writes both halves with 16-byte stores
// (conflict-free) into the plane's groups; after a CTA
// barrier one thread issues the 32 MMAs of the slab (P-1, P) and commits them
// to an mbarrier; each element warp reads its element's 24 outputs from its
// tensor-memory lane quadrant (warp w: element (w % 4, w / 4), lanes
// 32 (w % 4) .. + 31, columns 64 (w / 4) ..), scales them by E, and the corner
// contributions meet in k_lvl_op's exchange buffer and node phase (same fixed
// summation order). The TMA producer warp, stage ring and bounded waits are
// k_lvl_op's. 256 tensor-memory columns, allocated and freed by warp 0.
constexpr int kTcGroups = 5 * 4;                          // node-pair groups per plane: y 0..4, z 0..3
constexpr int kTcAtom = 1024;                             // one group: 32 realizations x 8 slots (bytes)
constexpr int kTcPlane = kTcGroups * kTcAtom;             // one half (hi or lo) of a plane
constexpr int kTcABytes = 2 * 2 * kTcPlane;               // planes P-1 and P, hi and lo: 80 KB
constexpr int kTcBFloats = 4 * 64 * 8;                    // 4 corner pairs x [B_hi | B_lo] (64) x 8 slots
constexpr int kTcCols = 256;                              // tensor-memory columns: 4 M tiles x 64
using TcStage = LvlStage<kLvlPcgZ>;
constexpr size_t kTcSmem = 1024 + kTcABytes + sizeof(float) * (kTcBFloats + (size_t)kMStages * TcStage::kFloats +
                                                                2 * (size_t)kMXFloats) +
                           sizeof(double) * kMJ * kMK * 32 + sizeof(uint64_t) * (2 * kMStages + 1) + 16;
static_assert(kTcSmem <= 227 * 1024, "tensor-core level operator shared memory");
static_assert((kTcABytes + sizeof(float) * kTcBFloats) % 128 == 0, "stage ring alignment");

__device__ __forceinline__ uint64_t tc_sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo, uint32_t layout) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | ((uint64_t)1 << 46) | ((uint64_t)(layout & 7u) << 61);
}
// instruction descriptor of kind::tf32: FP32 accumulator, A and B K-major
__device__ __forceinline__ uint32_t tc_idesc(int M, int N) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}
__device__ __forceinline__ void tc_mma(uint32_t tmem, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
  const uint32_t z = 0;
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem),
      "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(z), "r"(z), "r"(z), "r"(z));
}
__device__ __forceinline__ void tc_ld16(uint32_t a, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(a));
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tc_ld8(uint32_t a, float (&v)[8]) {
  uint32_t r[8];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
               : "r"(a));
#pragma unroll
  for (int i = 0; i < 8; ++i) v[i] = __uint_as_float(r[i]);
}
// byte offset of realization r's slots 0-3 in a 1 KB group (slots 4-7: + 128)
__device__ __forceinline__ uint32_t tc_row(int r) { return (uint32_t)((r >> 3) * 256 + (r & 7) * 16); }

template <int kMode>
__global__ void __launch_bounds__(kMThreads, 1)
    k_lvl_tc(Lattice L, const float* __restrict__ bops, const __grid_constant__ CUtensorMap tm_a,
             const __grid_constant__ CUtensorMap tm_b, const __grid_constant__ CUtensorMap tm_e,
             const __grid_constant__ CUtensorMap tm_d, int tiles_j, int n_tiles, int n_items,
             const uint8_t* __restrict__ mask, const float* __restrict__ alpha, const float* __restrict__ beta,
             float* __restrict__ out, float* __restrict__ out2, float* __restrict__ d, double* __restrict__ partial,
             int pstride, int* __restrict__ err) {
  static_assert(kMode == kLvlPcgZ, "the tensor-core level operator implements the search-direction launch");
  using S = TcStage;
  extern __shared__ __align__(1024) unsigned char tc_dyn[];
  unsigned char* base = tc_dyn + ((1024u - (smem_u32(tc_dyn) & 1023u)) & 1023u);
  unsigned char* abuf = base;                                             // [plane 2][hi, lo][group 20][1 KB]
  float* bsm = reinterpret_cast<float*>(base + kTcABytes);                // B operands
  float* smem = bsm + kTcBFloats;                                         // TMA stage ring
  float* xbuf = smem + kMStages * S::kFloats;
  double* red = reinterpret_cast<double*>(xbuf + 2 * kMXFloats);
  uint64_t* full = reinterpret_cast<uint64_t*>(red + kMJ * kMK * 32);
  uint64_t* empty = full + kMStages;
  uint64_t* mma_bar = empty + kMStages;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(mma_bar + 1);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int NX = L.NX, Rp = L.Rp;
  // zero both plane buffers (slots 6-7 stay zero), load the B operands
  for (int i = threadIdx.x; i < kTcABytes / 16; i += blockDim.x)
    reinterpret_cast<float4*>(abuf)[i] = make_float4(0.f, 0.f, 0.f, 0.f);
  for (int i = threadIdx.x; i < kTcBFloats / 4; i += blockDim.x)
    reinterpret_cast<float4*>(bsm)[i] = reinterpret_cast<const float4*>(bops)[i];
  if (threadIdx.x == 0) {
    for (int st = 0; st < kMStages; ++st) {
      mbar_init(&full[st], 1);
      mbar_init(&empty[st], kMWarps);
    }
    mbar_init(mma_bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (w == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(kTcCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;
  if (w == kMWarps) {  // TMA producer (k_lvl_op's)
    if (lane == 0) {
      uint32_t seq = 0;
      for (int item = blockIdx.x; item < n_items; item += gridDim.x) {
        const int tile = item % n_tiles, g32 = (item / n_tiles) * 32;
        const int J0 = 1 + (tile % tiles_j) * kMJ, K0 = 1 + (tile / tiles_j) * kMK;
        for (int P = 1; P <= NX; ++P, ++seq) {
          const int st = seq % kMStages;
          const uint32_t use = seq / kMStages;
          if (use > 0 && !mbar_wait(&empty[st], (use - 1) & 1)) {
            atomicExch(err, 1);
            return;
          }
          float* dst = smem + st * S::kFloats;
          mbar_expect_tx(&full[st], S::kBytes);
          tma_load_5d(dst + S::kOffA, &tm_a, g32, 0, P, J0 - 1, K0 - 1, &full[st]);
          tma_load_5d(dst + S::kOffB, &tm_b, g32, 0, P, J0 - 1, K0 - 1, &full[st]);
          tma_load_4d(dst + S::kOffE, &tm_e, g32, P - 1, J0 - 1, K0 - 1, &full[st]);
          tma_load_5d(dst + S::kOffD, &tm_d, g32, 0, P, J0, K0, &full[st]);
        }
      }
    }
    return;
  }
  const int ej = w % kMEJ, ek = w / kMEJ;
  const bool node_warp = ej >= 1 && ek >= 1;
  const uint32_t abase = smem_u32(abuf), bbase = smem_u32(bsm);
  // tensor-memory address of this warp's element: lanes 32 ej.., columns 64 ek..
  const uint32_t my_t = tmem + ((uint32_t)(32 * ej) << 16) + (uint32_t)(64 * ek);
  // node-pair groups this warp forms: (y = ej, z = ek), and the last element
  // column also (y = ej + 1, z = ek)
  const bool edge_y = ej == kMEJ - 1;
  uint32_t seq = 0, slab = 0;
  int xsel = 0;
  bool dead = false;
  auto csync = [&]() { asm volatile("bar.sync 1, %0;" ::"r"(kMWarps * 32) : "memory"); };
  for (int item = blockIdx.x; item < n_items; item += gridDim.x) {
    const int tile = item % n_tiles, g32 = (item / n_tiles) * 32;
    const int J0 = 1 + (tile % tiles_j) * kMJ, K0 = 1 + (tile / tiles_j) * kMK;
    const int Je = J0 - 1 + ej, Ke = K0 - 1 + ek;
    auto realj = [&](int j) { return j >= 1 && j <= L.NY - 1; };
    auto realk = [&](int k) { return k >= 1 && k <= L.NZ - 1; };
    const bool real = realj(Je) && realk(Ke);
    const bool node_ok = node_warp && Je <= L.NY && Ke <= L.NZ;
    const bool r00 = real, r10 = realj(Je - 1) && realk(Ke);
    const bool r01 = realj(Je) && realk(Ke - 1), r11 = realj(Je - 1) && realk(Ke - 1);
    const size_t nrow = ((size_t)Je + (size_t)L.NYp * Ke) * L.NXp;
    const int rr = g32 + lane;
    const float al = alpha[rr], be = beta[rr];
    float T0[12];  // corners (ay, az, c) of the plane below the slab being read, carried from the slab below it
#pragma unroll
    for (int i = 0; i < 12; ++i) T0[i] = 0.f;
    float ou[3] = {0.f, 0.f, 0.f};   // own node's p at the plane whose node phase runs next
    float ou1[3] = {0.f, 0.f, 0.f};  // ... and at the plane after it
    float E1 = 0.f;                  // E of the slab whose products are in flight
    double acc = 0.0;
    uint32_t mreg = 0;
    auto node_phase = [&](int X) {
      if (((X - 1) & 31) == 0) {
        const int pl = X + lane;
        mreg = (pl <= NX) ? mask[nrow + pl] : 0u;
      }
      const uint32_t mk = __shfl_sync(0xffffffffu, mreg, (X - 1) & 31);
      const float* xb = xbuf + xsel * kMXFloats;
      const size_t node = nrow + X;
      double sacc = 0.0;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        float y = 0.f;
        if (r00) y += xb[((w * 4 + 0) * 3 + c) * 32 + lane];
        if (r10) y += xb[(((w - 1) * 4 + 1) * 3 + c) * 32 + lane];
        if (r01) y += xb[(((w - kMEJ) * 4 + 2) * 3 + c) * 32 + lane];
        if (r11) y += xb[(((w - kMEJ - 1) * 4 + 3) * 3 + c) * 32 + lane];
        const size_t o = (node * 3 + c) * Rp + rr;
        const float v = ((mk >> c) & 1) ? 0.f : y;
        sacc = fma((double)ou[c], (double)v, sacc);
        out[o] = v;
      }
      acc += sacc;
    };
    auto emit_corners = [&]() {
      float* xb = xbuf + xsel * kMXFloats;
#pragma unroll
      for (int ay = 0; ay < 2; ++ay)
#pragma unroll
        for (int az = 0; az < 2; ++az)
#pragma unroll
          for (int c = 0; c < 3; ++c) xb[((w * 4 + ay + 2 * az) * 3 + c) * 32 + lane] = T0[(ay * 2 + az) * 3 + c];
    };
    // products of the slab committed last: wait, read this warp's element from
    // tensor memory, scale by its E (y: plane-below corners 0..11, plane-above 12..23)
    auto read_slab = [&](float (&y)[24]) {
      bool ok = !dead && mbar_wait(mma_bar, slab & 1);
      ++slab;
      ok = __all_sync(0xffffffffu, ok);
      if (!ok) {
        if (lane == 0) atomicExch(err, 1);
        dead = true;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      if (ok) {
        float a16[16], a8[8], b16[16], b8[8];
        tc_ld16(my_t, a16);
        tc_ld8(my_t + 16, a8);
        tc_ld16(my_t + 32, b16);
        tc_ld8(my_t + 48, b8);
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
        for (int i = 0; i < 16; ++i) y[i] = E1 * (a16[i] + b16[i]);
#pragma unroll
        for (int i = 0; i < 8; ++i) y[16 + i] = E1 * (a8[i] + b8[i]);
      } else {
#pragma unroll
        for (int i = 0; i < 24; ++i) y[i] = 0.f;
      }
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    };
    // corners of the slab's lower plane complete that plane: into the exchange
    // buffer (the node phase reads them after the next barrier)
    auto emit_slab = [&](const float (&y)[24]) {
      if (real) {
#pragma unroll
        for (int i = 0; i < 12; ++i) T0[i] += y[i];
        emit_corners();
      }
#pragma unroll
      for (int i = 0; i < 12; ++i) T0[i] = y[12 + i];
    };
    // Plane P: read the products of slab (P-2, P-1) (issued one plane earlier, so
    // they ran during the previous node phase) and emit plane P-2's corners, form
    // plane P into the buffer of plane P-2 (no longer read), and after one barrier
    // issue slab (P-1, P) into the same tensor memory (read above by every warp)
    // and run plane P-2's node phase.
    for (int P = 1; P <= NX; ++P, ++seq) {
      const int st = seq % kMStages;
      if (!dead && !mbar_wait(&full[st], (seq / kMStages) & 1)) {
        atomicExch(err, 1);
        dead = true;
      }
      const float* pt = smem + st * S::kFloats;
      if (P >= 3) {
        float y[24];
        read_slab(y);
        emit_slab(y);
      }
      // form p = z + beta p_old at the nodes of this warp's node-pair groups of plane P
      // (slots 0-2: node (y, z), 3-5: node (y, z + 1), 6-7: zero), split into hi and lo
      unsigned char* ap = abuf + (P & 1) * 2 * kTcPlane;
      float own[3] = {0.f, 0.f, 0.f};
#pragma unroll
      for (int f = 0; f < 2; ++f) {
        if (f == 1 && !edge_y) continue;
        const int py = ej + f, pz = ek;
        float u[6];
#pragma unroll
        for (int h = 0; h < 2; ++h)
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            const int i = (((pz + h) * kMPJ + py) * 3 + c) * 32 + lane;
            u[h * 3 + c] = fmaf(be, pt[S::kOffB + i], pt[S::kOffA + i]);
          }
        if (f == 0) {
          own[0] = u[0];
          own[1] = u[1];
          own[2] = u[2];
        }
        float hi[6], lo[6];
#pragma unroll
        for (int k = 0; k < 6; ++k) {
          hi[k] = __uint_as_float(__float_as_uint(u[k]) & 0xffffe000u);
          lo[k] = u[k] - hi[k];
        }
        unsigned char* g = ap + (uint32_t)(pz * 5 + py) * kTcAtom + tc_row(lane);
        *reinterpret_cast<float4*>(g) = make_float4(hi[0], hi[1], hi[2], hi[3]);
        *reinterpret_cast<float4*>(g + 128) = make_float4(hi[4], hi[5], 0.f, 0.f);
        *reinterpret_cast<float4*>(g + kTcPlane) = make_float4(lo[0], lo[1], lo[2], lo[3]);
        *reinterpret_cast<float4*>(g + kTcPlane + 128) = make_float4(lo[4], lo[5], 0.f, 0.f);
      }
      if (node_ok) {  // the owner writes p and d += alpha p_old (k_lvl_op<kLvlPcgZ>)
        const size_t node = nrow + P;
        const int op = ek * kMPJ + ej, od = (ek - 1) * kMJ + (ej - 1);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const size_t o = (node * 3 + c) * Rp + rr;
          const float pold = pt[S::kOffB + (op * 3 + c) * 32 + lane];
          out2[o] = own[c];
          d[o] = fmaf(al, pold, pt[S::kOffD + (od * 3 + c) * 32 + lane]);
        }
      }
      const float E = pt[S::kOffE + w * 32 + lane];
      __syncwarp();
      if (lane == 0) mbar_arrive(&empty[st]);
      // the plane's groups (generic-proxy writes) become visible to the tensor core
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      csync();
      if (P >= 2 && w == 0 && lane == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
        for (int t = 0; t < 4; ++t)      // M tile: the z row of element pencils
#pragma unroll
          for (int pr = 0; pr < 4; ++pr) {  // corner pair (ax, ay)
            const int ax = pr >> 1, ay = pr & 1;
            const uint32_t pa = abase + (uint32_t)((P - 1 + ax) & 1) * 2 * kTcPlane + (uint32_t)(t * 5 + ay) * kTcAtom;
            const uint32_t pb = bbase + (uint32_t)pr * 64 * 8 * 4;
            const uint64_t db = tc_sdesc(pb, 128, 256, 0);
            tc_mma(tmem + (uint32_t)(64 * t), tc_sdesc(pa, 128, 256, 0), db, tc_idesc(128, 64), pr > 0);
            tc_mma(tmem + (uint32_t)(64 * t), tc_sdesc(pa + kTcPlane, 128, 256, 0), db, tc_idesc(128, 32), 1u);
          }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                         smem_u32(mma_bar))
                     : "memory");
      }
      if (P >= 3) {
        if (node_ok) node_phase(P - 2);
        xsel ^= 1;
      }
      E1 = E;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        ou[c] = ou1[c];
        ou1[c] = own[c];
      }
    }
    // the last slab (NX-1, NX): plane NX-1, then plane NX from the carried corners
    {
      float y[24];
      read_slab(y);
      emit_slab(y);
    }
    csync();
    if (node_ok) node_phase(NX - 1);
    xsel ^= 1;
#pragma unroll
    for (int c = 0; c < 3; ++c) ou[c] = ou1[c];
    if (real) emit_corners();
    csync();
    if (node_ok) node_phase(NX);
    xsel ^= 1;
    if (partial != nullptr) {
      if (node_warp) red[((ek - 1) * kMJ + (ej - 1)) * 32 + lane] = acc;
      csync();
      if (w == 0) {
        double sum = 0.0;
#pragma unroll
        for (int i = 0; i < kMJ * kMK; ++i) sum += red[i * 32 + lane];
        partial[((size_t)tile * Rp + rr) * pstride] = sum;
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  csync();
  if (w == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTcCols));
  }
}

// ---------------------------------------------------------------- coarsest-level sweeps
// All damped Jacobi sweeps of the coarsest level in one launch. That level has
// at most 3 x 3 node pencils in (y, z), one k_lvl_op tile, so a CTA holds the
// whole level for its 32 realizations in shared memory (the iterate in two
// buffers, b, omega dinv, E and the mask, real nodes only) and consecutive
// sweeps are separated by CTA barriers instead of launches. Every sweep is the
// arithmetic of k_lvl_op<kLvlSmooth> in the same order (element warps over the
// x-planes, the same exchange and the same node sums), so the iterates are
// identical to the launch-per-sweep loop.
inline size_t coarse_sweep_smem(const Lattice& L) {
  const size_t nn = (size_t)L.NX * L.NY * L.NZ, ne = (size_t)(L.NX - 1) * (L.NY - 1) * (L.NZ - 1);
  return sizeof(float) * (nn * 32 * 10 + ne * 32 + 2 * (size_t)kMXFloats) + nn;
}
template <bool kMass>
__global__ void __launch_bounds__(kMWarps * 32, 1)
    k_coarse_sweeps(Lattice L, const __grid_constant__ ModalC C, const uint8_t* __restrict__ mask,
                    const float* __restrict__ b, const float* __restrict__ dinv, const float* __restrict__ E,
                    float omega, int n_sweeps, const float* __restrict__ x, float* __restrict__ out) {
  extern __shared__ __align__(16) float smem_cs[];
  const int NX = L.NX, NY = L.NY, NZ = L.NZ, Rp = L.Rp;
  const int nn = NX * NY * NZ, ne = (NX - 1) * (NY - 1) * (NZ - 1);
  float* src = smem_cs;           // iterate [node][c][32]
  float* dst = src + nn * 96;
  float* bs = dst + nn * 96;      // b [node][c][32]
  float* ws = bs + nn * 96;       // omega dinv [node][32]
  float* es = ws + nn * 32;       // E [element][32]
  float* xbuf = es + ne * 32;     // two exchange buffers
  uint8_t* mks = reinterpret_cast<uint8_t*>(xbuf + 2 * kMXFloats);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int rr = blockIdx.x * 32 + lane;
  auto cn = [&](int X, int J, int K) { return (X - 1) + NX * ((J - 1) + NY * (K - 1)); };
  auto ce = [&](int X, int J, int K) { return (X - 1) + (NX - 1) * ((J - 1) + (NY - 1) * (K - 1)); };
  auto pn = [&](int X, int J, int K) { return (size_t)X + (size_t)L.NXp * ((size_t)J + (size_t)L.NYp * K); };
  for (int i = w; i < nn; i += kMWarps) {
    const int X = i % NX + 1, J = (i / NX) % NY + 1, K = i / (NX * NY) + 1;
    const size_t pi = pn(X, J, K);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      src[(i * 3 + c) * 32 + lane] = x[(pi * 3 + c) * Rp + rr];
      bs[(i * 3 + c) * 32 + lane] = b[(pi * 3 + c) * Rp + rr];
    }
    ws[i * 32 + lane] = omega * dinv[pi * Rp + rr];
    if (lane == 0) mks[i] = mask[pi];
  }
  for (int i = w; i < ne; i += kMWarps) {
    const int X = i % (NX - 1) + 1, J = (i / (NX - 1)) % (NY - 1) + 1, K = i / ((NX - 1) * (NY - 1)) + 1;
    es[i * 32 + lane] = E[pn(X, J, K) * Rp + rr];
  }
  __syncthreads();
  // the tile starts at node pencil (1, 1): element pencil (Je, Ke) = (ej, ek)
  const int Je = w % kMEJ, Ke = w / kMEJ;
  auto realj = [&](int j) { return j >= 1 && j <= NY - 1; };
  auto realk = [&](int k) { return k >= 1 && k <= NZ - 1; };
  const bool real = realj(Je) && realk(Ke);
  const bool node_ok = Je >= 1 && Ke >= 1 && Je <= NY && Ke <= NZ;
  const bool r00 = real, r10 = realj(Je - 1) && realk(Ke);
  const bool r01 = realj(Je) && realk(Ke - 1), r11 = realj(Je - 1) && realk(Ke - 1);
  int xsel = 0;
  for (int sw = 0; sw < n_sweeps; ++sw) {
    float Bp[3][4], T0[3][4], ou[3] = {0.f, 0.f, 0.f};
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int qq = 0; qq < 4; ++qq) T0[c][qq] = 0.f;
    auto node_phase = [&](int X) {
      const int i = cn(X, Je, Ke);
      const uint32_t mk = mks[i];
      const float* xb = xbuf + xsel * kMXFloats;
      const float wdv = ws[i * 32 + lane];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        float y = 0.f;
        if (r00) y += xb[((w * 4 + 0) * 3 + c) * 32 + lane];
        if (r10) y += xb[(((w - 1) * 4 + 1) * 3 + c) * 32 + lane];
        if (r01) y += xb[(((w - kMEJ) * 4 + 2) * 3 + c) * 32 + lane];
        if (r11) y += xb[(((w - kMEJ - 1) * 4 + 3) * 3 + c) * 32 + lane];
        const float bv = bs[(i * 3 + c) * 32 + lane];
        dst[(i * 3 + c) * 32 + lane] = ((mk >> c) & 1) ? 0.f : fmaf(wdv, bv - y, ou[c]);
      }
    };
    auto emit_corners = [&](const float (&B)[3][4]) {
      float y[2][2][3];
      yz_inverse(B, y);
      float* xb = xbuf + xsel * kMXFloats;
#pragma unroll
      for (int ay = 0; ay < 2; ++ay)
#pragma unroll
        for (int az = 0; az < 2; ++az)
#pragma unroll
          for (int c = 0; c < 3; ++c) xb[((w * 4 + ay + 2 * az) * 3 + c) * 32 + lane] = y[ay][az][c];
    };
    for (int P = 1; P <= NX; ++P) {
      float u[2][2][3];
#pragma unroll
      for (int ay = 0; ay < 2; ++ay)
#pragma unroll
        for (int az = 0; az < 2; ++az) {
          const int J = Je + ay, K = Ke + az;
          const bool in = J >= 1 && J <= NY && K >= 1 && K <= NZ;  // ghost nodes are zero
          const int i = in ? cn(P, J, K) : 0;
#pragma unroll
          for (int c = 0; c < 3; ++c) u[ay][az][c] = in ? src[(i * 3 + c) * 32 + lane] : 0.f;
        }
      float Bc[3][4];
      yz_forward(u, Bc);
      if (P >= 2) {
        if (real) {
          float C1[3][4];
          modal_apply<kMass>(C, es[ce(P - 1, Je, Ke) * 32 + lane], Bp, Bc, T0, C1);
          emit_corners(T0);
#pragma unroll
          for (int c = 0; c < 3; ++c)
#pragma unroll
            for (int qq = 0; qq < 4; ++qq) T0[c][qq] = C1[c][qq];
        }
        __syncthreads();
        if (node_ok) node_phase(P - 1);
        xsel ^= 1;
      }
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        ou[c] = u[0][0][c];
#pragma unroll
        for (int qq = 0; qq < 4; ++qq) Bp[c][qq] = Bc[c][qq];
      }
    }
    if (real) emit_corners(T0);
    __syncthreads();
    if (node_ok) node_phase(NX);
    xsel ^= 1;
    __syncthreads();  // the sweep's iterate is complete before the next one reads it
    float* tmp = src;
    src = dst;
    dst = tmp;
  }
  for (int i = w; i < nn; i += kMWarps) {
    const int X = i % NX + 1, J = (i / NX) % NY + 1, K = i / (NX * NY) + 1;
    const size_t pi = pn(X, J, K);
#pragma unroll
    for (int c = 0; c < 3; ++c) out[(pi * 3 + c) * Rp + rr] = src[(i * 3 + c) * 32 + lane];
  }
}

// ---------------------------------------------------------------- packed level operator (level 0)
// k_lvl_op with two realizations per lane in float2 registers: the element and
// node arithmetic issues Blackwell's packed FP32 instructions (one issue slot
// for both), halving the instructions per realization of an issue-bound
// kernel. A 3 x 3 tile of node pencils with its 16 element warps for 64
// realizations, at most 128 registers a thread (16 warps fill the register
// file: 4 warps per SM sub-partition), and no separate producer warp: lane 0
// of warp 0 issues the TMA loads two planes ahead (the 3-stage ring refills
// the stage of the plane before the current one; its readers have arrived on
// its "empty" barrier, a bounded wait). The exchange buffer holds corners 1..3
// of each element (corner 0 stays in the registers of the warp that owns its
// node pencil), which leaves room for the 5 x 5 node patches. Modes, barriers
// and bounded waits as k_lvl_op otherwise.
constexpr int kQJ = 3, kQK = 3;                     // node pencils per tile (y, z)
constexpr int kQEJ = kQJ + 1, kQEK = kQK + 1;       // element pencils 4 x 4
constexpr int kQWarps = kQEJ * kQEK;                // 16 element warps
constexpr int kQThreads = 32 * kQWarps;
constexpr int kQPJ = kQJ + 2, kQPK = kQK + 2;       // node patch 5 x 5
constexpr int kQR = 64;                             // realizations per work item
constexpr int kQPlane = kQR * 3 * kQPJ * kQPK;      // vector patch (floats)
constexpr int kQNode = kQR * kQPJ * kQPK;           // dinv patch
constexpr int kQE = kQR * kQEJ * kQEK;              // E patch
constexpr int kQD = kQR * 3 * kQJ * kQK;            // d of the tile's own nodes
// exchange buffer: corners 1..3 of every element warp (corner 0 belongs to the
// node pencil of the warp itself and stays in its registers)
constexpr int kQX = kQWarps * 3 * 3 * kQR;
template <int kMode> struct LvlStage2 {
  static constexpr bool kTwo = kMode == kLvlStart || kMode == kLvlPcgZ;
  // Smooth and Resid also stage b of the tile's own nodes (Smooth its dinv as
  // well), read by the node phase one plane later: their stages are released
  // after that node phase, so the ring has 4 stages (loads still go two planes ahead)
  static constexpr bool kOwn = kMode == kLvlSmooth || kMode == kLvlResid;
  static constexpr bool kOwnD = kMode == kLvlSmooth;
  static constexpr int kStages = kOwn ? 4 : kMStages;
  static constexpr int kOffA = 0;
  static constexpr int kOffB = kQPlane;
  static constexpr int kOffN = (kTwo ? 2 : 1) * kQPlane;
  static constexpr int kOffE = kOffN + (kMode == kLvlStart ? kQNode : 0);
  static constexpr int kOffD = kOffE + kQE;  // d (direction) or own b (smooth, resid)
  static constexpr int kOffO = kOffD + (kOwn ? kQD : 0);  // own dinv (smooth)
  static constexpr int kFloats = kOffO + (kMode == kLvlPcgZ ? kQD : 0) + (kOwnD ? kQR * kQJ * kQK : 0);
  static constexpr uint32_t kBytes = kFloats * 4;
  static constexpr size_t kSmem = 128 + sizeof(float) * ((size_t)kStages * kFloats + 2 * (size_t)kQX) +
                                  sizeof(double) * kQJ * kQK * kQR + sizeof(uint64_t) * (2 * kStages);
};
static_assert(LvlStage2<kLvlStart>::kBytes % 128 == 0 && LvlStage2<kLvlSmooth>::kBytes % 128 == 0 &&
                  LvlStage2<kLvlPcgZ>::kBytes % 128 == 0 && LvlStage2<kLvlResid>::kBytes % 128 == 0 &&
                  LvlStage2<kLvlResid>::kSmem <= 227 * 1024,
              "stage alignment");
static_assert(LvlStage2<kLvlPcgZ>::kSmem <= 227 * 1024 && LvlStage2<kLvlStart>::kSmem <= 227 * 1024 &&
                  LvlStage2<kLvlSmooth>::kSmem <= 227 * 1024 && (kQR * kQJ * kQK * 4) % 128 == 0,
              "smem");

template <int kMode, bool kMass>
__global__ void __maxnreg__(128)
    k_lvl_op2(Lattice L, const __grid_constant__ ModalCT<float2> C, const __grid_constant__ CUtensorMap tm_a,
              const __grid_constant__ CUtensorMap tm_b, const __grid_constant__ CUtensorMap tm_n,
              const __grid_constant__ CUtensorMap tm_e, const __grid_constant__ CUtensorMap tm_d, int tiles_j,
              int n_tiles, int n_items, const uint8_t* __restrict__ mask, const float* __restrict__ b,
              const float* __restrict__ dinv, float omega, const float* __restrict__ alpha,
              const float* __restrict__ beta, float* __restrict__ out, float* __restrict__ out2,
              float* __restrict__ out3, float* __restrict__ d, double* __restrict__ partial, int pstride,
              int* __restrict__ err) {
  using S = LvlStage2<kMode>;
  extern __shared__ __align__(128) float smem_dyn[];
  float* smem = smem_dyn + (((128u - (smem_u32(smem_dyn) & 127u)) & 127u) >> 2);
  constexpr int kSt = S::kStages;
  float* xbuf = smem + kSt * S::kFloats;
  double* red = reinterpret_cast<double*>(xbuf + 2 * kQX);  // [node pencils][64]
  uint64_t* full = reinterpret_cast<uint64_t*>(red + kQJ * kQK * kQR);
  uint64_t* empty = full + kSt;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int NX = L.NX, Rp = L.Rp, Rp2 = L.Rp >> 1;
  if (threadIdx.x == 0) {
    for (int st = 0; st < kSt; ++st) {
      mbar_init(&full[st], 1);
      mbar_init(&empty[st], kQWarps);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  // producer role: global step q loads (item, plane) = (blockIdx.x + (q / NX) gridDim.x, q % NX + 1)
  // into stage q % 3
  const bool producer = w == 0 && lane == 0;
  auto produce = [&](uint32_t q) {
    const int item = blockIdx.x + (int)(q / (uint32_t)NX) * gridDim.x;
    if (item >= n_items) return;
    const int P = (int)(q % (uint32_t)NX) + 1;
    const int tile = item % n_tiles, g64 = (item / n_tiles) * kQR;
    const int J0 = 1 + (tile % tiles_j) * kQJ, K0 = 1 + (tile / tiles_j) * kQK;
    const int st = q % kSt;
    const uint32_t use = q / kSt;
    if (use > 0 && !mbar_wait(&empty[st], (use - 1) & 1)) {
      atomicExch(err, 1);
      return;
    }
    float* dst = smem + st * S::kFloats;
    mbar_expect_tx(&full[st], S::kBytes);
    tma_load_5d(dst + S::kOffA, &tm_a, g64, 0, P, J0 - 1, K0 - 1, &full[st]);
    if constexpr (S::kTwo) tma_load_5d(dst + S::kOffB, &tm_b, g64, 0, P, J0 - 1, K0 - 1, &full[st]);
    if constexpr (kMode == kLvlStart) tma_load_4d(dst + S::kOffN, &tm_n, g64, P, J0 - 1, K0 - 1, &full[st]);
    tma_load_4d(dst + S::kOffE, &tm_e, g64, P - 1, J0 - 1, K0 - 1, &full[st]);
    if constexpr (kMode == kLvlPcgZ) tma_load_5d(dst + S::kOffD, &tm_d, g64, 0, P, J0, K0, &full[st]);
    if constexpr (S::kOwn) tma_load_5d(dst + S::kOffD, &tm_b, g64, 0, P, J0, K0, &full[st]);
    if constexpr (S::kOwnD) tma_load_4d(dst + S::kOffO, &tm_n, g64, P, J0, K0, &full[st]);
  };
  if (producer) {
    produce(0);
    produce(1);
  }
  const int ej = w % kQEJ, ek = w / kQEJ;
  const bool node_warp = ej >= 1 && ek >= 1;
  uint32_t seq = 0;
  int xsel = 0;
  bool dead = false;
  auto csync = [&]() { asm volatile("bar.sync 1, %0;" ::"r"(kQWarps * 32) : "memory"); };
  const float2 z2 = make_float2(0.f, 0.f);
  for (int item = blockIdx.x; item < n_items; item += gridDim.x) {
    const int tile = item % n_tiles, g64 = (item / n_tiles) * kQR;
    const int J0 = 1 + (tile % tiles_j) * kQJ, K0 = 1 + (tile / tiles_j) * kQK;
    const int Je = J0 - 1 + ej, Ke = K0 - 1 + ek;
    auto realj = [&](int j) { return j >= 1 && j <= L.NY - 1; };
    auto realk = [&](int k) { return k >= 1 && k <= L.NZ - 1; };
    const bool real = realj(Je) && realk(Ke);
    const bool node_ok = node_warp && Je <= L.NY && Ke <= L.NZ;
    const bool r00 = real, r10 = realj(Je - 1) && realk(Ke);
    const bool r01 = realj(Je) && realk(Ke - 1), r11 = realj(Je - 1) && realk(Ke - 1);
    const size_t nrow = ((size_t)Je + (size_t)L.NYp * Ke) * L.NXp;
    const int rr2 = (g64 >> 1) + lane;  // float2 index of this lane's realization pair
    float2 al = z2, be = z2;
    if constexpr (kMode == kLvlStart || kMode == kLvlPcgZ) al = reinterpret_cast<const float2*>(alpha)[rr2];
    if constexpr (kMode == kLvlPcgZ) be = reinterpret_cast<const float2*>(beta)[rr2];
    const float2 nal = make_float2(-al.x, -al.y);
    const float2 om2 = make_float2(omega, omega);
    const float2* xb2 = reinterpret_cast<const float2*>(xbuf);
    float2* out_2 = reinterpret_cast<float2*>(out);
    float2 Bp[3][4], T0[3][4];
    float2 ou[3] = {z2, z2, z2}, orc[3] = {z2, z2, z2};
    float2 own[3] = {z2, z2, z2};  // corner 0 of the warp's element: its own node pencil
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int qq = 0; qq < 4; ++qq) T0[c][qq] = z2;
    double acc0 = 0.0, acc1 = 0.0;
    uint32_t mreg = 0;
    auto node_phase = [&](int X, uint32_t seq_x) {
      [[maybe_unused]] const float* px = smem + (seq_x % kSt) * S::kFloats;
      [[maybe_unused]] const int od = (ek - 1) * kQJ + (ej - 1);
      if (((X - 1) & 31) == 0) {
        const int pl = X + lane;
        mreg = (pl <= NX) ? mask[nrow + pl] : 0u;
      }
      const uint32_t mk = __shfl_sync(0xffffffffu, mreg, (X - 1) & 31);
      const float2* xb = xb2 + xsel * (kQX / 2);
      const size_t node = nrow + X;
      float2 wdv = z2;
      if constexpr (kMode == kLvlSmooth) wdv = om2 * reinterpret_cast<const float2*>(px + S::kOffO)[od * 32 + lane];
      double s0 = 0.0, s1 = 0.0;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        float2 y = z2;
        if (r00) y = y + own[c];
        if (r10) y = y + xb[(((w - 1) * 3 + 0) * 3 + c) * 32 + lane];
        if (r01) y = y + xb[(((w - kQEJ) * 3 + 1) * 3 + c) * 32 + lane];
        if (r11) y = y + xb[(((w - kQEJ - 1) * 3 + 2) * 3 + c) * 32 + lane];
        const size_t o = (node * 3 + c) * Rp2 + rr2;
        const bool fixed = (mk >> c) & 1;
        float2 v;
        if constexpr (kMode == kLvlStart) {
          v = fixed ? z2 : orc[c] - y;
          s0 = fma((double)orc[c].x, (double)orc[c].x, s0);
          s1 = fma((double)orc[c].y, (double)orc[c].y, s1);
        } else if constexpr (kMode == kLvlResid) {
          v = fixed ? z2 : reinterpret_cast<const float2*>(px + S::kOffD)[(od * 3 + c) * 32 + lane] - y;
        } else if constexpr (kMode == kLvlSmooth) {
          const float2 bv = reinterpret_cast<const float2*>(px + S::kOffD)[(od * 3 + c) * 32 + lane];
          v = fixed ? z2 : fmx(wdv, bv - y, ou[c]);
          s0 = fma((double)v.x, (double)bv.x, s0);
          s1 = fma((double)v.y, (double)bv.y, s1);
        } else {
          v = fixed ? z2 : y;
          s0 = fma((double)ou[c].x, (double)v.x, s0);
          s1 = fma((double)ou[c].y, (double)v.y, s1);
        }
        out_2[o] = v;
      }
      acc0 += s0;
      acc1 += s1;
    };
    auto emit_corners = [&](const float2 (&B)[3][4]) {
      float2 y[2][2][3];
      yz_inverse(B, y);
      float2* xb = reinterpret_cast<float2*>(xbuf) + xsel * (kQX / 2);
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        own[c] = y[0][0][c];
        xb[((w * 3 + 0) * 3 + c) * 32 + lane] = y[1][0][c];
        xb[((w * 3 + 1) * 3 + c) * 32 + lane] = y[0][1][c];
        xb[((w * 3 + 2) * 3 + c) * 32 + lane] = y[1][1][c];
      }
    };
    for (int P = 1; P <= NX; ++P, ++seq) {
      const int st = seq % kSt;
      if (producer && !dead) produce(seq + 2);
      if (!dead && !mbar_wait(&full[st], (seq / kSt) & 1)) {
        atomicExch(err, 1);
        dead = true;
      }
      const float* pt = smem + st * S::kFloats;
      const float2* pa = reinterpret_cast<const float2*>(pt + S::kOffA);
      const float2* pb = reinterpret_cast<const float2*>(pt + S::kOffB);
      float2 u[2][2][3], rc[3] = {z2, z2, z2};
#pragma unroll
      for (int ay = 0; ay < 2; ++ay)
#pragma unroll
        for (int az = 0; az < 2; ++az) {
          const int o = (ek + az) * kQPJ + (ej + ay);
          float2 wdv = z2;
          if constexpr (kMode == kLvlStart)
            wdv = om2 * reinterpret_cast<const float2*>(pt + S::kOffN)[o * 32 + lane];
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            const int i = (o * 3 + c) * 32 + lane;
            if constexpr (kMode == kLvlStart) {
              const float2 rn = fmx(nal, pb[i], pa[i]);
              u[ay][az][c] = wdv * rn;
              if (ay == 0 && az == 0) rc[c] = rn;
            } else if constexpr (kMode == kLvlPcgZ) {
              u[ay][az][c] = fmx(be, pb[i], pa[i]);
            } else {
              u[ay][az][c] = pa[i];
            }
          }
        }
      const float2 E = reinterpret_cast<const float2*>(pt + S::kOffE)[w * 32 + lane];
      if constexpr (kMode == kLvlStart || kMode == kLvlPcgZ) {
        if (node_ok) {
          const size_t node = nrow + P;
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            const size_t o = (node * 3 + c) * Rp2 + rr2;
            if constexpr (kMode == kLvlStart) {
              reinterpret_cast<float2*>(out2)[o] = rc[c];
              if (out3 != nullptr) reinterpret_cast<float2*>(out3)[o] = u[0][0][c];
            } else {
              const int op = ek * kQPJ + ej, od = (ek - 1) * kQJ + (ej - 1);
              const float2 pold = pb[(op * 3 + c) * 32 + lane];
              const float2 dold = reinterpret_cast<const float2*>(pt + S::kOffD)[(od * 3 + c) * 32 + lane];
              reinterpret_cast<float2*>(out2)[o] = u[0][0][c];
              reinterpret_cast<float2*>(d)[o] = fmx(al, pold, dold);
            }
          }
        }
      }
      __syncwarp();
      if (!S::kOwn && lane == 0) mbar_arrive(&empty[st]);
      float2 Bc[3][4];
      yz_forward(u, Bc);
      if (P >= 2) {
        if (real) {
          float2 C1[3][4];
          modal_apply<kMass>(C, E, Bp, Bc, T0, C1);
          emit_corners(T0);
#pragma unroll
          for (int c = 0; c < 3; ++c)
#pragma unroll
            for (int qq = 0; qq < 4; ++qq) T0[c][qq] = C1[c][qq];
        }
        csync();
        if (node_ok) node_phase(P - 1, seq - 1);
        xsel ^= 1;
        if constexpr (S::kOwn) {  // the node phase of plane P - 1 is done with its stage
          __syncwarp();
          if (lane == 0) mbar_arrive(&empty[(seq - 1) % kSt]);
        }
      }
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        ou[c] = u[0][0][c];
        orc[c] = rc[c];
#pragma unroll
        for (int qq = 0; qq < 4; ++qq) Bp[c][qq] = Bc[c][qq];
      }
    }
    if (real) emit_corners(T0);
    csync();
    if (node_ok) node_phase(NX, seq - 1);
    xsel ^= 1;
    if constexpr (S::kOwn) {
      __syncwarp();
      if (lane == 0) mbar_arrive(&empty[(seq - 1) % kSt]);
    }
    if (kMode != kLvlResid && partial != nullptr) {
      if (node_warp) {
        const int nw = (ek - 1) * kQJ + (ej - 1);
        red[nw * kQR + 2 * lane] = acc0;
        red[nw * kQR + 2 * lane + 1] = acc1;
      }
      csync();
      if (w < 2) {
        const int rl = w * 32 + lane;  // realization within the item
        double sum = 0.0;
#pragma unroll
        for (int i = 0; i < kQJ * kQK; ++i) sum += red[i * kQR + rl];
        partial[((size_t)tile * Rp + g64 + rl) * pstride] = sum;
      }
    }
  }
}

// ---------------------------------------------------------------- FP64 true residual (Walsh modes)
// The reliable-update step of the batched loops in one pass: with kUpdate the
// corner input is x + d + alpha p (the FP32 correction folded into the FP64
// iterate; the owner writes the new x into the other x buffer; d is cleared
// after the launch, since neighbouring tiles read it in their halos), otherwise x; then r = b - A x in FP64 with the Walsh-mode operator (mass term
// with kMass), masked, r32 = (float) r, and the per-realization partials
// ||r||^2, dinv r32.r32 ([tile][Rp][2], the layout of k_resid). A CTA owns a
// 3 x 2 tile of node pencils with its 12 element warps (FP64 element state
// needs about twice the registers of the FP32 operator: 3 warps per SM
// sub-partition) and no separate producer warp: lane 0 of warp 0 issues the
// TMA loads three planes ahead into the 4-stage ring (refilling the stage of
// the plane before the current one, a bounded wait on its "empty" barrier);
// exchange and bounded waits as k_op_modal.
constexpr int kRJ = 3, kRK = 2;
constexpr int kREJ = kRJ + 1, kREK = kRK + 1, kRWarps = kREJ * kREK;
constexpr int kRPJ = kRJ + 2, kRPK = kRK + 2;
constexpr int kRThreads = 32 * kRWarps;
constexpr int kRPatch = 32 * 3 * kRPJ * kRPK;          // values of a vector patch (1536)
constexpr int kREPatch = 32 * kREJ * kREK;             // E patch (288 doubles)
constexpr uint32_t kROffX = 0, kROffD = 8 * kRPatch, kROffP = kROffD + 4 * kRPatch, kROffE = kROffP + 4 * kRPatch;
constexpr uint32_t kRStageBytes = kROffE + 8 * kREPatch;  // 33,792 bytes
constexpr int kRStages = 4;
constexpr int kRXDoubles = kRWarps * 4 * 3 * 32;        // exchange buffer (doubles)
constexpr size_t kRSmem = 128 + (size_t)kRStages * kRStageBytes + 2 * sizeof(double) * kRXDoubles +
                          sizeof(double) * 2 * kRJ * kRK * 32 + sizeof(uint64_t) * (2 * kRStages);
static_assert(kRStageBytes % 128 == 0 && kROffD % 128 == 0 && kROffP % 128 == 0 && kROffE % 128 == 0, "align");
static_assert(kRSmem <= 227 * 1024, "FP64 residual shared memory");

template <bool kMass, bool kBPerR, bool kUpdate>
__global__ void __launch_bounds__(kRThreads, 1)
    k_resid_modal(Lattice L, const __grid_constant__ ModalCD C, const __grid_constant__ CUtensorMap tm_x,
                  const __grid_constant__ CUtensorMap tm_d, const __grid_constant__ CUtensorMap tm_p,
                  const __grid_constant__ CUtensorMap tm_e, int tiles_j, int n_tiles, int n_items,
                  const uint8_t* __restrict__ mask, const double* __restrict__ b, const float* __restrict__ dinv,
                  const float* __restrict__ alpha, double* __restrict__ x_out, float* __restrict__ r32,
                  double* __restrict__ partial, int* __restrict__ err) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  unsigned char* smem = smem_raw + ((128u - (smem_u32(smem_raw) & 127u)) & 127u);
  double* xbuf = reinterpret_cast<double*>(smem + (size_t)kRStages * kRStageBytes);
  double* red = xbuf + 2 * kRXDoubles;  // [2][node pencils][32]
  uint64_t* full = reinterpret_cast<uint64_t*>(red + 2 * kRJ * kRK * 32);
  uint64_t* empty = full + kRStages;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int NX = L.NX, Rp = L.Rp;
  constexpr uint32_t kBytes = kUpdate ? kRStageBytes : (8 * kRPatch + 8 * kREPatch);
  if (threadIdx.x == 0) {
    for (int st = 0; st < kRStages; ++st) {
      mbar_init(&full[st], 1);
      mbar_init(&empty[st], kRWarps);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  // producer role: global step q loads (item, plane) = (blockIdx.x + (q / NX) gridDim.x, q % NX + 1)
  const bool producer = w == 0 && lane == 0;
  auto produce = [&](uint32_t q) {
    const int item = blockIdx.x + (int)(q / (uint32_t)NX) * gridDim.x;
    if (item >= n_items) return;
    const int P = (int)(q % (uint32_t)NX) + 1;
    const int tile = item % n_tiles, g32 = (item / n_tiles) * 32;
    const int J0 = 1 + (tile % tiles_j) * kRJ, K0 = 1 + (tile / tiles_j) * kRK;
    const int st = q % kRStages;
    const uint32_t use = q / kRStages;
    if (use > 0 && !mbar_wait(&empty[st], (use - 1) & 1)) {
      atomicExch(err, 1);
      return;
    }
    unsigned char* dst = smem + (size_t)st * kRStageBytes;
    mbar_expect_tx(&full[st], kBytes);
    tma_load_5d(dst + kROffX, &tm_x, g32, 0, P, J0 - 1, K0 - 1, &full[st]);
    if constexpr (kUpdate) {
      tma_load_5d(dst + kROffD, &tm_d, g32, 0, P, J0 - 1, K0 - 1, &full[st]);
      tma_load_5d(dst + kROffP, &tm_p, g32, 0, P, J0 - 1, K0 - 1, &full[st]);
    }
    tma_load_4d(dst + (kUpdate ? kROffE : 8 * kRPatch), &tm_e, g32, P - 1, J0 - 1, K0 - 1, &full[st]);
  };
  if (producer)
    for (int q = 0; q < kRStages - 1; ++q) produce(q);
  const int ej = w % kREJ, ek = w / kREJ;
  const bool node_warp = ej >= 1 && ek >= 1;
  uint32_t seq = 0;
  int xsel = 0;
  bool dead = false;
  auto csync = [&]() { asm volatile("bar.sync 1, %0;" ::"r"(kRWarps * 32) : "memory"); };
  for (int item = blockIdx.x; item < n_items; item += gridDim.x) {
    const int tile = item % n_tiles, g32 = (item / n_tiles) * 32;
    const int J0 = 1 + (tile % tiles_j) * kRJ, K0 = 1 + (tile / tiles_j) * kRK;
    const int Je = J0 - 1 + ej, Ke = K0 - 1 + ek;
    auto realj = [&](int j) { return j >= 1 && j <= L.NY - 1; };
    auto realk = [&](int k) { return k >= 1 && k <= L.NZ - 1; };
    const bool real = realj(Je) && realk(Ke);
    const bool node_ok = node_warp && Je <= L.NY && Ke <= L.NZ;
    const bool r00 = real, r10 = realj(Je - 1) && realk(Ke);
    const bool r01 = realj(Je) && realk(Ke - 1), r11 = realj(Je - 1) && realk(Ke - 1);
    const size_t nrow = ((size_t)Je + (size_t)L.NYp * Ke) * L.NXp;
    const int rr = g32 + lane;
    double al = 0.0;
    if constexpr (kUpdate) al = (double)alpha[rr];
    double Bp[3][4], T0[3][4];
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int qq = 0; qq < 4; ++qq) T0[c][qq] = 0.0;
    double acc_rr = 0.0, acc_dz = 0.0;
    uint32_t mreg = 0;
    // b and dinv of the node the next node phase completes, loaded one plane
    // ahead so that their latency hides behind the element work
    double nb[3] = {0.0, 0.0, 0.0};
    float ndv = 0.f;
    auto prefetch = [&](int X) {
      if (!node_ok) return;
      const size_t node = nrow + X;
      ndv = dinv[node * Rp + rr];
#pragma unroll
      for (int c = 0; c < 3; ++c) nb[c] = kBPerR ? b[(node * 3 + c) * Rp + rr] : b[node * 3 + c];
    };
    auto node_phase = [&](int X) {
      if (((X - 1) & 31) == 0) {
        const int pl = X + lane;
        mreg = (pl <= NX) ? mask[nrow + pl] : 0u;
      }
      const uint32_t mk = __shfl_sync(0xffffffffu, mreg, (X - 1) & 31);
      const double* xb = xbuf + xsel * kRXDoubles;
      const size_t node = nrow + X;
      const double dv = (double)ndv;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        double y = 0.0;
        if (r00) y += xb[((w * 4 + 0) * 3 + c) * 32 + lane];
        if (r10) y += xb[(((w - 1) * 4 + 1) * 3 + c) * 32 + lane];
        if (r01) y += xb[(((w - kREJ) * 4 + 2) * 3 + c) * 32 + lane];
        if (r11) y += xb[(((w - kREJ - 1) * 4 + 3) * 3 + c) * 32 + lane];
        const size_t o = (node * 3 + c) * Rp + rr;
        const double bv = nb[c];
        const double rc = ((mk >> c) & 1) ? 0.0 : bv - y;
        const float rf = (float)rc;
        r32[o] = rf;
        acc_rr = fma(rc, rc, acc_rr);
        acc_dz = fma(dv * (double)rf, (double)rf, acc_dz);
      }
    };
    auto emit_corners = [&](const double (&B)[3][4]) {
      double y[2][2][3];
      yz_inverse(B, y);
      double* xb = xbuf + xsel * kRXDoubles;
#pragma unroll
      for (int ay = 0; ay < 2; ++ay)
#pragma unroll
        for (int az = 0; az < 2; ++az)
#pragma unroll
          for (int c = 0; c < 3; ++c) xb[((w * 4 + ay + 2 * az) * 3 + c) * 32 + lane] = y[ay][az][c];
    };
    for (int P = 1; P <= NX; ++P, ++seq) {
      const int st = seq % kRStages;
      if (producer && !dead) produce(seq + kRStages - 1);
      if (!dead && !mbar_wait(&full[st], (seq / kRStages) & 1)) {
        atomicExch(err, 1);
        dead = true;
      }
      if (P >= 2) prefetch(P - 1);
      const unsigned char* pt = smem + (size_t)st * kRStageBytes;
      const double* px = reinterpret_cast<const double*>(pt + kROffX);
      const float* pd = reinterpret_cast<const float*>(pt + kROffD);
      const float* pp = reinterpret_cast<const float*>(pt + kROffP);
      const double* pe = reinterpret_cast<const double*>(pt + (kUpdate ? kROffE : 8 * kRPatch));
      double u[2][2][3];
#pragma unroll
      for (int ay = 0; ay < 2; ++ay)
#pragma unroll
        for (int az = 0; az < 2; ++az) {
          const int o = (ek + az) * kRPJ + (ej + ay);
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            const int i = (o * 3 + c) * 32 + lane;
            double v = px[i];
            if constexpr (kUpdate) v += (double)pd[i] + al * (double)pp[i];
            u[ay][az][c] = v;
          }
        }
      const double E = pe[w * 32 + lane];
      if constexpr (kUpdate) {
        if (node_ok) {
          const size_t node = nrow + P;
#pragma unroll
          for (int c = 0; c < 3; ++c) x_out[(node * 3 + c) * Rp + rr] = u[0][0][c];
        }
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(&empty[st]);
      double Bc[3][4];
      yz_forward(u, Bc);
      if (P >= 2) {
        if (real) {
          double C1[3][4];
          modal_apply<kMass>(C, E, Bp, Bc, T0, C1);
          emit_corners(T0);
#pragma unroll
          for (int c = 0; c < 3; ++c)
#pragma unroll
            for (int qq = 0; qq < 4; ++qq) T0[c][qq] = C1[c][qq];
        }
        csync();
        if (node_ok) node_phase(P - 1);
        xsel ^= 1;
      }
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int qq = 0; qq < 4; ++qq) Bp[c][qq] = Bc[c][qq];
    }
    prefetch(NX);
    if (real) emit_corners(T0);
    csync();
    if (node_ok) node_phase(NX);
    xsel ^= 1;
    if (node_warp) {
      const int nw = (ek - 1) * kRJ + (ej - 1);
      red[(0 * kRJ * kRK + nw) * 32 + lane] = acc_rr;
      red[(1 * kRJ * kRK + nw) * 32 + lane] = acc_dz;
    }
    csync();
    if (w < 2) {
      double sum = 0.0;
#pragma unroll
      for (int i = 0; i < kRJ * kRK; ++i) sum += red[(w * kRJ * kRK + i) * 32 + lane];
      partial[((size_t)tile * Rp + rr) * 2 + w] = sum;
    }
  }
}

// Full-weighting restriction b_c = P^T t_f (P: trilinear prolongation), masked
// at the coarse level, and x_c = omega dinv_c b_c (the first Jacobi sweep from
// zero). Coarse node (I, J, K) (padded) sits on fine node (2I-1, 2J-1, 2K-1);
// the fine ghost layer is zero. Grid: x = coarse interior node, y = chunks of
// 128 float4 realization groups; one thread per node and four realizations.
// Offsets are 32-bit and relative to the centre node (the 27 loads of a
// component share one base address).
constexpr int kXferThreads = 128;
constexpr int kProlongNodes = 2;  // fine nodes of one k_prolong_add CTA
__global__ void __launch_bounds__(kXferThreads, 8) k_restrict(Lattice Lf, Lattice Lc, const int* __restrict__ interior_c,
                                                              const uint8_t* __restrict__ mask_c,
                                                              const float* __restrict__ tf,
                                                              const float* __restrict__ dinv_c, float omega,
                                                              float* __restrict__ bc, float* __restrict__ xc) {
  const int Q = Lf.Rp >> 2;
  const int q = blockIdx.y * kXferThreads + threadIdx.x;
  if (q >= Q) return;
  const int nc = interior_c[blockIdx.x];
  const int I = nc % Lc.NXp, J = (nc / Lc.NXp) % Lc.NYp, K = nc / (Lc.NXp * Lc.NYp);
  const int fc = (2 * I - 1) + Lf.NXp * ((2 * J - 1) + Lf.NYp * (2 * K - 1));
  const int sx = 3 * Q, sy = Lf.NXp * sx, sz = Lf.NYp * sy;  // float4 strides between fine nodes
  const float4* t4 = reinterpret_cast<const float4*>(tf) + (size_t)fc * sx + q;
  const uint32_t mk = mask_c[nc];
  const size_t oc = (size_t)nc * sx + q;
  const float4* dv4 = reinterpret_cast<const float4*>(dinv_c) + (size_t)nc * Q + q;
  float4* b4 = reinterpret_cast<float4*>(bc) + oc;
  float4* x4 = reinterpret_cast<float4*>(xc) + oc;
#pragma unroll 1
  for (int c = 0; c < 3; ++c) {
    float4 s = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
    for (int dz = -1; dz <= 1; ++dz)
#pragma unroll
      for (int dy = -1; dy <= 1; ++dy)
#pragma unroll
        for (int dx = -1; dx <= 1; ++dx) {
          const float wgt = (dx ? 0.5f : 1.f) * (dy ? 0.5f : 1.f) * (dz ? 0.5f : 1.f);
          const float4 v = t4[dx * sx + dy * sy + dz * sz + c * Q];
          s.x = fmaf(wgt, v.x, s.x);
          s.y = fmaf(wgt, v.y, s.y);
          s.z = fmaf(wgt, v.z, s.z);
          s.w = fmaf(wgt, v.w, s.w);
        }
    if ((mk >> c) & 1) s = make_float4(0.f, 0.f, 0.f, 0.f);
    b4[c * Q] = s;
    const float4 dv = *dv4;  // loaded after the sums: no register held across the 27 loads
    x4[c * Q] = make_float4(omega * dv.x * s.x, omega * dv.y * s.y, omega * dv.z * s.z, omega * dv.w * s.w);
  }
}

// x_f += P x_c: trilinear prolongation of the coarse correction (per axis, a
// fine node with even coordinate takes the coincident coarse node, an odd one
// the mean of its two neighbours), masked at the fine level. Grid as
// k_restrict over the fine interior nodes; the 8 corner terms are summed in a
// fixed order (the terms of an even axis's second neighbour, weight 0, are skipped).
// With r0 given, the iterate before the correction is not read from x_f but
// formed as the first Jacobi sweep from zero, x0 = (omega dinv0) r0, with the
// arithmetic of the start pass (which then need not write it), and x_f is
// written at every component (the constrained ones without the correction).
__global__ void __launch_bounds__(kXferThreads, 8) k_prolong_add(Lattice Lf, Lattice Lc,
                                                                 const int* __restrict__ interior_f, int n_int,
                                                                 const uint8_t* __restrict__ mask_f,
                                                                 const float* __restrict__ xc, float* __restrict__ xf,
                                                                 const float* __restrict__ r0,
                                                                 const float* __restrict__ dinv0, float omega) {
  const int Q = Lf.Rp >> 2;
  const int q = blockIdx.y * kXferThreads + threadIdx.x;
  if (q >= Q) return;
  const int sx = 3 * Q, sy = Lc.NXp * sx, sz = Lc.NYp * sy;  // float4 strides between coarse nodes
  // kProlongNodes fine nodes a CTA, their loads in flight together
#pragma unroll
  for (int u = 0; u < kProlongNodes; ++u) {
    const int t = blockIdx.x * kProlongNodes + u;
    if (t >= n_int) break;
    const int nf = interior_f[t];
    const uint32_t mk = mask_f[nf];
    if (mk == 7u && r0 == nullptr) continue;
    const int gi = nf % Lf.NXp - 1, gj = (nf / Lf.NXp) % Lf.NYp - 1, gk = nf / (Lf.NXp * Lf.NYp) - 1;
    const int c0 = ((gi >> 1) + 1) + Lc.NXp * (((gj >> 1) + 1) + Lc.NYp * ((gk >> 1) + 1));
    const int oi = (gi & 1) * sx, oj = (gj & 1) * sy, ok = (gk & 1) * sz;  // offset of the second neighbour (or 0)
    const float wi[2] = {(gi & 1) ? 0.5f : 1.f, (gi & 1) ? 0.5f : 0.f};
    const float wj[2] = {(gj & 1) ? 0.5f : 1.f, (gj & 1) ? 0.5f : 0.f};
    const float wk[2] = {(gk & 1) ? 0.5f : 1.f, (gk & 1) ? 0.5f : 0.f};
    const float4* c4 = reinterpret_cast<const float4*>(xc) + (size_t)c0 * sx + q;
    float4* f4 = reinterpret_cast<float4*>(xf) + (size_t)nf * sx + q;
    float4 wdv = make_float4(0.f, 0.f, 0.f, 0.f);
    if (r0 != nullptr) {
      const float4 dv = reinterpret_cast<const float4*>(dinv0)[(size_t)nf * Q + q];
      wdv = make_float4(omega * dv.x, omega * dv.y, omega * dv.z, omega * dv.w);
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      float4 s;
      if (r0 != nullptr) {
        const float4 rv = reinterpret_cast<const float4*>(r0)[((size_t)nf * 3 + c) * Q + q];
        s = make_float4(wdv.x * rv.x, wdv.y * rv.y, wdv.z * rv.z, wdv.w * rv.w);
        if ((mk >> c) & 1) {
          f4[c * Q] = s;
          continue;
        }
      } else {
        if ((mk >> c) & 1) continue;
        s = f4[c * Q];
      }
#pragma unroll
      for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int bb = 0; bb < 2; ++bb)
#pragma unroll
          for (int e = 0; e < 2; ++e) {
            // an even coordinate has one coarse neighbour on that axis: skip the zero-weight loads
            if ((e && !(gi & 1)) || (bb && !(gj & 1)) || (a && !(gk & 1))) continue;
            const float wgt = wk[a] * wj[bb] * wi[e];
            const float4 v = c4[(e ? oi : 0) + (bb ? oj : 0) + (a ? ok : 0) + c * Q];
            s.x = fmaf(wgt, v.x, s.x);
            s.y = fmaf(wgt, v.y, s.y);
            s.z = fmaf(wgt, v.z, s.z);
            s.w = fmaf(wgt, v.w, s.w);
          }
      f4[c * Q] = s;
    }
  }
}

// grid of the transfer kernels: x = interior node, y = chunks of kXferThreads float4 groups
inline dim3 xfer_grid(int n_int, int Rp) {
  return dim3((unsigned)n_int, (unsigned)((Rp / 4 + kXferThreads - 1) / kXferThreads));
}
inline int xfer_block(int Rp) { return std::min(kXferThreads, (Rp / 4 + 31) / 32 * 32); }
inline dim3 prolong_grid(int n_int, int Rp) {
  return dim3((unsigned)((n_int + kProlongNodes - 1) / kProlongNodes),
              (unsigned)((Rp / 4 + kXferThreads - 1) / kXferThreads));
}

// Coarse element field: the mean of the 8 fine elements it covers (elements
// are stored at their lower-corner padded node). One CTA per coarse element.
__global__ void __launch_bounds__(128) k_coarsen_E(Lattice Lf, Lattice Lc, int nxc, int nyc,
                                                   const float* __restrict__ Ef, float* __restrict__ Ec) {
  const int e = blockIdx.x;
  const int I = e % nxc + 1, J = (e / nxc) % nyc + 1, K = e / (nxc * nyc) + 1;
  const size_t nc = (size_t)I + (size_t)Lc.NXp * (J + (size_t)Lc.NYp * K);
  const size_t sy = (size_t)Lf.NXp, sz = (size_t)Lf.NXp * Lf.NYp;
  const size_t f0 = (size_t)(2 * I - 1) + sy * (2 * J - 1) + sz * (2 * K - 1);
  const int Rp = Lf.Rp;
  for (int rr = threadIdx.x; rr < Rp; rr += blockDim.x) {
    double s = 0.0;
    for (int a = 0; a < 2; ++a)
      for (int bb = 0; bb < 2; ++bb)
        for (int c = 0; c < 2; ++c) s += (double)Ef[(f0 + c + bb * sy + a * sz) * Rp + rr];
    Ec[nc * Rp + rr] = (float)(0.125 * s);
  }
}

// FP64 operator application y (+)= (E Khat + Mhat on real elements) x, no
// mask, batch layout (the Newmark right-hand side).
template <bool kAccumulate>
__global__ void __launch_bounds__(128)
    k_apply64(Lattice L, const __grid_constant__ KhatD K, const __grid_constant__ MassClasses<double> M,
              const double* __restrict__ x, const double* __restrict__ E, double* __restrict__ y) {
  int J, Kz;
  bool valid;
  pencil_of(L, J, Kz, valid);
  const int Rp = L.Rp;
  const int rr = blockIdx.y * 32 + threadIdx.x;
  if (!valid) return;
  auto emit = [&](size_t node, const double*, const double* v) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      double* o = y + (node * 3 + c) * Rp + rr;
      *o = kAccumulate ? *o + v[c] : v[c];
    }
  };
  auto load = [&](size_t node, double* o) {
#pragma unroll
    for (int c = 0; c < 3; ++c) o[c] = ldv(x + (node * 3 + c) * Rp + rr);
  };
  auto own = [](size_t, const double*) {};
  pencil_sweep<double, true>(L, K, J, Kz, E + rr, load, own, emit, &M);
}

// Jacobi diagonal: A_nn,cc = Khat_diag * sum of E over the node's 8 elements
// (all 24 diagonal entries of a cube's Khat are equal) + Mhat_diag * the
// number of real elements (E > 0) around the node; 0 on ghosts.
__global__ void k_dinv(Lattice L, double kdiag, double mdiag, const float* __restrict__ E,
                       const int* __restrict__ interior, float* __restrict__ dinv) {
  const int t = blockIdx.x;
  const size_t node = (size_t)interior[t];
  const size_t sxy = (size_t)L.NXp, sxz = (size_t)L.NXp * L.NYp;
  for (int rr = threadIdx.x; rr < L.Rp; rr += blockDim.x) {
    double s = 0;
    int n_real = 0;
    for (int ez = -1; ez <= 0; ++ez)
      for (int ey = -1; ey <= 0; ++ey)
        for (int ex = -1; ex <= 0; ++ex) {
          const float e = E[(node + ex + ey * sxy + ez * sxz) * L.Rp + rr];
          s += (double)e;
          n_real += e > 0.f;
        }
    dinv[node * L.Rp + rr] = (float)(1.0 / (kdiag * s + mdiag * n_real));
  }
}

struct Scal {
  float* alpha;        // [Rp]
  float* beta;         // [Rp]
  double* gamma;       // [Rp] (dinv r).r
  double* gamma_prev;  // [Rp] gamma of the previous iteration
  double* rho_ref;     // [Rp] r.r (gamma for the single-reduction loop) at the last reliable update
  double* res;         // [Rp] FP64 ||b - K x|| / ||b||
  double* bnorm;       // [Rp]
  double* gamma0;      // [Rp] gamma of the first true residual (r = b)
  int* act;            // [Rp] iterating
  int* done;           // [Rp] converged (true residual)
  int* its;            // [Rp] operator applications
  int* breakdown;      // [Rp] 1: PCG breakdown, 2: iteration limit of the slot reached
  int* fresh;          // [Rp] 1: the slot starts a new system at the next true-residual step
  int* n_active;       // [1] active count after the last k_beta / k_resid_scalars
  int* n_update;       // [1] active realizations requesting a reliable update
  int* err;            // [1] sticky: a bounded device wait expired
};

// Per-realization sum of NV interleaved partials over n rows, 32 realizations x
// 32 row-groups per CTA; fixed summation order (row-group sequential, then the
// 32 groups in order), so results are reproducible and independent of the batch.
template <int NV>
__device__ __forceinline__ void reduce_rows(const double* __restrict__ partial, int n, int Rp, double (&out)[NV]) {
  __shared__ double sh[32][NV][33];
  const int lane = threadIdx.x & 31, g = threadIdx.x >> 5;
  const int r = blockIdx.x * 32 + lane;
  double acc[NV];
#pragma unroll
  for (int q = 0; q < NV; ++q) acc[q] = 0.0;
  for (int t = g; t < n; t += 32)
#pragma unroll
    for (int q = 0; q < NV; ++q) acc[q] += partial[((size_t)t * Rp + r) * NV + q];
#pragma unroll
  for (int q = 0; q < NV; ++q) sh[g][q][lane] = acc[q];
  __syncthreads();
#pragma unroll
  for (int q = 0; q < NV; ++q) {
    double s = 0.0;
#pragma unroll 4
    for (int gg = 0; gg < 32; ++gg) s += sh[gg][q][lane];
    out[q] = s;
  }
}

// After a true-residual replacement: convergence test, new reference norm and
// the search-direction coefficient beta = gamma_new / gamma_prev (first call:
// beta = 0, p starts from z). gamma_ref: 0 two-reduction Jacobi loop (reference
// norm r.r), 1 single-reduction loop ((dinv r).r), 2 multigrid loop (r.r; beta
// is left to k_gmg_beta).
__global__ void __launch_bounds__(1024) k_resid_scalars(int Rp, int n_tiles, const double* __restrict__ partial,
                                                        Scal s, double tol, int first, int gamma_ref, int max_it) {
  double v[2];
  reduce_rows<2>(partial, n_tiles, Rp, v);
  const int r = blockIdx.x * 32 + threadIdx.x;
  int active = 0;
  if (threadIdx.x < 32) {
    const double rr = v[0], g = v[1];
    const double bn = s.bnorm[r];
    const double rel = bn > 0 ? sqrt(rr) / bn : 0.0;
    const int fr = first || s.fresh[r];
    s.fresh[r] = 0;
    s.res[r] = rel;
    if (!s.done[r] && (bn <= 1e-25 || rel < tol)) s.done[r] = 1;
    if (!s.done[r] && !s.breakdown[r] && s.its[r] >= max_it) s.breakdown[r] = 2;
    const int a = (s.done[r] || s.breakdown[r]) ? 0 : 1;
    s.act[r] = a;
    if (gamma_ref == 2) {
      // multigrid loop: beta follows from the next preconditioned residual
      // (k_gmg_beta); a fresh system starts its direction from z
      if (fr) s.gamma_prev[r] = 0.0;
    } else {
      s.beta[r] = (a && !fr && s.gamma_prev[r] > 0) ? (float)(g / s.gamma_prev[r]) : 0.f;
      s.gamma[r] = g;
    }
    s.rho_ref[r] = gamma_ref == 1 ? g : rr;
    s.alpha[r] = 0.f;  // the pending alpha p term was folded into x (and no r update is pending)
    active = a;
  }
  active = __syncthreads_count(active);
  if (threadIdx.x == 0 && active) atomicAdd(s.n_active, active);
}

// Scalars of the single-reduction loop after k_op_modal: with gamma = (dinv r).r
// of the launch's r, alpha = gamma / p.q, gamma' = gamma - 2 alpha (dinv r).q +
// alpha^2 q.dinv.q (the gamma of the next r), beta = gamma' / gamma;
// a reliable update is requested once gamma has dropped by delta^2 since the
// last one, or below tol2 * gamma0.
__global__ void __launch_bounds__(1024) k_alpha_gamma(int Rp, int n_tiles, const double* __restrict__ partial, Scal s,
                                                      double delta2, double tol2) {
  double v[4];
  reduce_rows<4>(partial, n_tiles, Rp, v);
  const int r = blockIdx.x * 32 + threadIdx.x;
  int active = 0, upd = 0;
  if (threadIdx.x < 32) {
    float a = 0.f, b = 0.f;
    if (s.act[r]) {
      const double pq = v[0], zq = v[1], qdq = v[2], g = v[3];
      const double al = g / pq;
      double gn = g - 2.0 * al * zq + al * al * qdq;
      if (g == 0.0) {
        // the recursive residual vanished: hold still and ask for a true-residual check
        active = 1;
        upd = 1;
      } else if (!(pq > 0.0) || !(g > 0.0) || !(gn == gn)) {
        s.act[r] = 0;
        s.breakdown[r] = 1;
      } else {
        gn = gn > 0.0 ? gn : 0.0;  // rounding at convergence; the true residual decides
        a = (float)al;
        b = (float)(gn / g);
        s.its[r] += 1;
        s.gamma_prev[r] = g;
        s.gamma[r] = gn;
        active = 1;
        upd = (gn < delta2 * s.rho_ref[r] || gn < tol2 * s.gamma0[r]) ? 1 : 0;
      }
    }
    s.alpha[r] = a;
    s.beta[r] = b;
  }
  active = __syncthreads_count(active);
  upd = __syncthreads_count(upd);
  if (threadIdx.x == 0) {
    if (active) atomicAdd(s.n_active, active);
    if (upd) atomicAdd(s.n_update, upd);
  }
}

// Scalars of the multigrid-preconditioned loop after the level-0 post-smoothing:
// partials [tile][Rp][2] = (r'.r', z.r') with r' the updated residual and z = M r'.
// gamma = z.r', beta = gamma / gamma_prev (0 after a fresh start), and a
// reliable update is requested once r'.r' has dropped by delta^2 since the last
// one or below tol2 * ||b||^2. A vanished residual holds the realization still
// until the true-residual check.
__global__ void __launch_bounds__(1024) k_gmg_beta(int Rp, int n_tiles, const double* __restrict__ partial, Scal s,
                                                   double delta2, double tol2) {
  double v[2];
  reduce_rows<2>(partial, n_tiles, Rp, v);
  const int r = blockIdx.x * 32 + threadIdx.x;
  int active = 0, upd = 0;
  if (threadIdx.x < 32) {
    float b = 0.f;
    if (s.act[r]) {
      const double rr = v[0], zr = v[1];
      if (rr == 0.0) {
        s.gamma[r] = 0.0;
        active = 1;
        upd = 1;
      } else if (!(zr > 0.0) || !(rr == rr)) {
        s.act[r] = 0;
        s.breakdown[r] = 1;
      } else {
        const double gp = s.gamma_prev[r];
        b = gp > 0.0 ? (float)(zr / gp) : 0.f;
        s.gamma[r] = zr;
        s.gamma_prev[r] = zr;
        active = 1;
        const double bn = s.bnorm[r];
        upd = (rr < delta2 * s.rho_ref[r] || rr < tol2 * bn * bn) ? 1 : 0;
      }
    }
    s.beta[r] = b;
  }
  active = __syncthreads_count(active);
  upd = __syncthreads_count(upd);
  if (threadIdx.x == 0) {
    if (active) atomicAdd(s.n_active, active);
    if (upd) atomicAdd(s.n_update, upd);
  }
}

// alpha = gamma / p.(A p) of the multigrid loop; a held realization (gamma = 0)
// keeps alpha = 0.
__global__ void __launch_bounds__(1024) k_gmg_alpha(int Rp, int n_tiles, const double* __restrict__ partial, Scal s) {
  double v[1];
  reduce_rows<1>(partial, n_tiles, Rp, v);
  if (threadIdx.x >= 32) return;
  const int r = blockIdx.x * 32 + threadIdx.x;
  const double pq = v[0];
  float a = 0.f;
  if (s.act[r] && s.gamma[r] > 0.0) {
    if (!(pq > 0.0)) {
      s.act[r] = 0;
      s.breakdown[r] = 1;
    } else {
      a = (float)(s.gamma[r] / pq);
      s.its[r] += 1;
    }
  }
  s.alpha[r] = a;
}

// Per-realization ||b||^2 and (dinv b).b of a batch right-hand side (shared
// vector b[node*3 + c] or, with per_r, the batch layout): CTA partials
// [blk][Rp][2] over a slice of the interior nodes (32 realizations x 8 groups).
__global__ void __launch_bounds__(256) k_bsq(int n_int, int Rp, const int* __restrict__ interior,
                                             const double* __restrict__ b, int per_r, const float* __restrict__ dinv,
                                             double* __restrict__ partial) {
  __shared__ double sh[8][2][32];
  const int lane = threadIdx.x & 31, g = threadIdx.x >> 5;
  const int rr = blockIdx.y * 32 + lane;
  const int per = (n_int + gridDim.x - 1) / gridDim.x;
  const int t0 = blockIdx.x * per, t1 = min(n_int, t0 + per);
  double a = 0.0, z = 0.0;
  for (int t = t0 + g; t < t1; t += 8) {
    const size_t n = (size_t)interior[t];
    const double dv = (double)dinv[n * Rp + rr];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const double v = per_r ? b[(n * 3 + c) * Rp + rr] : b[n * 3 + c];
      a += v * v;
      z += dv * v * v;
    }
  }
  sh[g][0][lane] = a;
  sh[g][1][lane] = z;
  __syncthreads();
  if (g == 0) {
    double sa = 0.0, sz = 0.0;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      sa += sh[k][0][lane];
      sz += sh[k][1][lane];
    }
    partial[((size_t)blockIdx.x * Rp + rr) * 2] = sa;
    partial[((size_t)blockIdx.x * Rp + rr) * 2 + 1] = sz;
  }
}

// bnorm = ||b|| and gamma0 = (dinv b).b per realization (0 beyond R)
__global__ void __launch_bounds__(1024) k_bnorm(int R, int Rp, int n_blk, const double* __restrict__ partial, Scal s) {
  double v[2];
  reduce_rows<2>(partial, n_blk, Rp, v);
  const int r = blockIdx.x * 32 + threadIdx.x;
  if (threadIdx.x < 32) {
    s.bnorm[r] = r < R ? sqrt(v[0]) : 0.0;
    s.gamma0[r] = r < R ? v[1] : 0.0;
  }
}

// Newmark right-hand-side inputs (interior nodes, batch layout):
// w1 = c1u u + c1v v + c1a a (mass part), w2 = c2u u + c2v v + c2a a (stiffness part)
__global__ void k_nm_pre(int n_int, int Rp, const int* __restrict__ interior, const double* __restrict__ u,
                         const double* __restrict__ v, const double* __restrict__ a, double c1u, double c1v,
                         double c1a, double c2u, double c2v, double c2a, double* __restrict__ w1,
                         double* __restrict__ w2) {
  const size_t total = (size_t)n_int * 3 * Rp;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    const size_t row = i / Rp;
    const size_t o = ((size_t)interior[row / 3] * 3 + row % 3) * Rp + (i - row * Rp);
    const double uu = c1u * u[o] + c1v * v[o] + c1a * a[o];
    const double uc = c2u * u[o] + c2v * v[o] + c2a * a[o];
    w1[o] = uu;
    w2[o] = uc;
  }
}

// y = (free rows) y + f_static + ag * fM, 0 on constrained rows
__global__ void k_nm_rhs(int n_int, int Rp, const int* __restrict__ interior, const uint8_t* __restrict__ mask,
                         const double* __restrict__ f_static, const double* __restrict__ fM, double ag,
                         double* __restrict__ y) {
  const size_t total = (size_t)n_int * 3 * Rp;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    const size_t row = i / Rp;
    const size_t node = (size_t)interior[row / 3];
    const int c = (int)(row % 3);
    const size_t o = (node * 3 + c) * Rp + (i - row * Rp);
    const double f = (f_static ? f_static[node * 3 + c] : 0.0) + ag * fM[node * 3 + c];
    y[o] = ((mask[node] >> c) & 1) ? 0.0 : y[o] + f;
  }
}

// after the solve x of step i: a' = a0 (x - u) - a2 v - a3 a, v += a6 a + a7 a', u = x
__global__ void k_nm_post(int n_int, int Rp, const int* __restrict__ interior, const double* __restrict__ x,
                          double* __restrict__ u, double* __restrict__ v, double* __restrict__ a, double a0,
                          double a2, double a3, double a6, double a7) {
  const size_t total = (size_t)n_int * 3 * Rp;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    const size_t row = i / Rp;
    const size_t o = ((size_t)interior[row / 3] * 3 + row % 3) * Rp + (i - row * Rp);
    const double an = a0 * (x[o] - u[o]) - a2 * v[o] - a3 * a[o];
    v[o] += a6 * a[o] + a7 * an;
    a[o] = an;
    u[o] = x[o];
  }
}

// start of a Newmark step's solve: the Newmark predictor x = u + dt v + (1/2 - alpha) dt^2 a
// (elementwise over the whole batch layout; padding and constrained entries stay 0)
__global__ void k_nm_predict(size_t n, const double* __restrict__ u, const double* __restrict__ v,
                             const double* __restrict__ a, double cv, double ca, double* __restrict__ x) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    x[i] = u[i] + cv * v[i] + ca * a[i];
}

// unit vector field: component dir = 1 at every interior node (batch layout)
__global__ void k_unit_dir(int n_int, int Rp, const int* __restrict__ interior, int dir, double* __restrict__ e) {
  const size_t total = (size_t)n_int * Rp;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    const size_t t = i / Rp;
    e[((size_t)interior[t] * 3 + dir) * Rp + (i - t * Rp)] = 1.0;
  }
}

// one realization's column of a batch-layout vector into a shared vector
__global__ void k_column(size_t n, int Rp, int r, const double* __restrict__ a, double* __restrict__ b) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    b[i] = a[i * Rp + r];
}

// Serving slots: zero the batch-vector columns of the listed realization
// slots and reset their scalars (fresh: the next true-residual step starts a
// new system there).
__global__ void k_slot_reset(int n_slots, const int* __restrict__ slots, size_t nrows, int Rp, double* __restrict__ x,
                             float* __restrict__ v0, float* __restrict__ v1, float* __restrict__ v2,
                             float* __restrict__ v3, float* __restrict__ v4, float* __restrict__ v5,
                             float* __restrict__ v6, Scal s) {
  const size_t total = (size_t)n_slots * nrows;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    const size_t row = i % nrows;
    const size_t o = row * Rp + slots[i / nrows];
    x[o] = 0.0;
    v0[o] = v1[o] = v2[o] = v3[o] = v4[o] = v5[o] = v6[o] = 0.f;
  }
  const size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (t < (size_t)n_slots) {
    const int r = slots[t];
    s.alpha[r] = s.beta[r] = 0.f;
    s.gamma[r] = s.gamma_prev[r] = s.rho_ref[r] = s.res[r] = 0.0;
    s.act[r] = s.done[r] = s.its[r] = s.breakdown[r] = 0;
    s.fresh[r] = 1;
  }
}

// Jacobi diagonal (as k_dinv) for the listed slots only
__global__ void k_dinv_slots(Lattice L, double kdiag, double mdiag, const float* __restrict__ E,
                             const int* __restrict__ interior, int n_slots, const int* __restrict__ slots,
                             float* __restrict__ dinv) {
  const size_t node = (size_t)interior[blockIdx.x];
  const size_t sxy = (size_t)L.NXp, sxz = (size_t)L.NXp * L.NYp;
  for (int i = threadIdx.x; i < n_slots; i += blockDim.x) {
    const int rr = slots[i];
    double s = 0;
    int n_real = 0;
    for (int ez = -1; ez <= 0; ++ez)
      for (int ey = -1; ey <= 0; ++ey)
        for (int ex = -1; ex <= 0; ++ex) {
          const float e = E[(node + ex + ey * sxy + ez * sxz) * L.Rp + rr];
          s += (double)e;
          n_real += e > 0.f;
        }
    dinv[node * L.Rp + rr] = (float)(1.0 / (kdiag * s + mdiag * n_real));
  }
}

// out[dof] = x[row(dof)*Rp + slot]
__global__ void k_gather_column(int n_dofs, int Rp, int slot, const int* __restrict__ rows,
                                const double* __restrict__ x, double* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n_dofs) out[i] = x[(size_t)rows[i] * Rp + slot];
}

__global__ void k_fill_int(int* __restrict__ a, int n, int v) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) a[i] = v;
}

__global__ void k_lattice_rhs(int n_dofs, const int* __restrict__ rows, const double* __restrict__ b_dof,
                              double* __restrict__ b_lat) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n_dofs) b_lat[rows[i]] = b_dof[i];
}

// r32 = (float) b over the interior nodes (b shared, b[node*3 + c], or per
// realization in the batch layout); constrained entries of b are zero.
__global__ void __launch_bounds__(256) k_b_to_r32(int n_int, int Rp, const int* __restrict__ interior,
                                                  const double* __restrict__ b, int per_r, float* __restrict__ r32) {
  const long total = (long)n_int * Rp;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
    const int t = (int)(i / Rp), rr = (int)(i % Rp);
    const size_t node = (size_t)interior[t];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const size_t o = (node * 3 + c) * Rp + rr;
      r32[o] = (float)(per_r ? b[o] : b[node * 3 + c]);
    }
  }
}

// X[r][dof] = x[(row(dof))*Rp + r] through a 32x32 shared-memory transpose.
__global__ void k_gather_solution(int n_dofs, int R, int Rp, const int* __restrict__ rows,
                                  const double* __restrict__ x, double* __restrict__ X) {
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

__global__ void k_gather_tip(int R, int Rp, int row, const double* __restrict__ x, double* __restrict__ tip) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r < R) tip[r] = x[(size_t)row * Rp + r];
}

__global__ void k_f64_to_f32(size_t n, const double* __restrict__ a, float* __restrict__ b) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    b[i] = (float)a[i];
}

// Walsh-mode form of a cube's element matrices (host, FP64): Km = T^T K T with
// T = s (x) I3. Fills the block coefficients of cK * Khat / 64 (and the
// diagonal of cM * Mhat / 64 when M576 is given) and checks that every other
// entry vanishes, so the modal operator reproduces the element matrices.
int modal_coefficients(Context* ctx, const double* K576, const double* M576, double cK, double cM, ModalC* out,
                       ModalCD* out64 = nullptr) {
  auto sgn = [](int a, int m) {  // s(a, m) for corner id a and mode m
    const int ax = (a == 1 || a == 2 || a == 5 || a == 6), ay = (a == 2 || a == 3 || a == 6 || a == 7), az = a >= 4;
    int s = 1;
    if ((m & 1) && !ax) s = -s;
    if ((m & 2) && !ay) s = -s;
    if ((m & 4) && !az) s = -s;
    return s;
  };
  auto to_modal = [&](const double* A, std::vector<double>& Am) {
    Am.assign(576, 0.0);
    for (int m = 0; m < 8; ++m)
      for (int c = 0; c < 3; ++c)
        for (int m2 = 0; m2 < 8; ++m2)
          for (int c2 = 0; c2 < 3; ++c2) {
            double s = 0;
            for (int a = 0; a < 8; ++a)
              for (int b = 0; b < 8; ++b) s += sgn(a, m) * sgn(b, m2) * A[(3 * a + c) * 24 + 3 * b + c2];
            Am[(3 * m + c) * 24 + 3 * m2 + c2] = s;
          }
  };
  std::vector<double> Km;
  to_modal(K576, Km);
  auto at = [&](int m, int c, int m2, int c2) { return Km[(3 * m + c) * 24 + 3 * m2 + c2]; };
  const double va = at(1, 0, 1, 0), vb = at(1, 0, 2, 1), sa = at(1, 1, 1, 1), sb = at(1, 1, 2, 0);
  const double pa = at(3, 0, 3, 0), pb = at(3, 0, 6, 2), ta = at(3, 2, 3, 2), tb = at(3, 2, 5, 1);
  const double da = at(7, 0, 7, 0);
  // rebuild Km from the nine blocks
  std::vector<double> R(576, 0.0);
  auto put_block = [&](std::initializer_list<std::pair<int, int>> dofs, double a, double b) {
    for (auto i : dofs)
      for (auto j : dofs) R[(3 * i.first + i.second) * 24 + 3 * j.first + j.second] = (i == j) ? a : b;
  };
  put_block({{1, 0}, {2, 1}, {4, 2}}, va, vb);
  put_block({{1, 1}, {2, 0}}, sa, sb);
  put_block({{1, 2}, {4, 0}}, sa, sb);
  put_block({{2, 2}, {4, 1}}, sa, sb);
  put_block({{3, 0}, {6, 2}}, pa, pb);
  put_block({{3, 1}, {5, 2}}, pa, pb);
  put_block({{5, 0}, {6, 1}}, pa, pb);
  put_block({{3, 2}, {5, 1}, {6, 0}}, ta, tb);
  put_block({{7, 0}}, da, 0.0);
  put_block({{7, 1}}, da, 0.0);
  put_block({{7, 2}}, da, 0.0);
  double kmax = 0, dev = 0;
  for (int i = 0; i < 576; ++i) {
    kmax = std::max(kmax, std::fabs(Km[i]));
    dev = std::max(dev, std::fabs(Km[i] - R[i]));
  }
  if (!(dev <= 1e-11 * kmax))
    return set_error(ctx, MSG_ERR_NOT_STRUCTURED, "element stiffness lacks the cube's modal structure (%g)", dev / kmax);
  const double f = cK / 64.0;
  out->vd = (float)((va - vb) * f);
  out->vb = (float)(vb * f);
  out->sa = (float)(sa * f);
  out->sb = (float)(sb * f);
  out->pa = (float)(pa * f);
  out->pb = (float)(pb * f);
  out->td = (float)((ta - tb) * f);
  out->tb = (float)(tb * f);
  out->da = (float)(da * f);
  for (int m = 0; m < 8; ++m) out->m[m] = 0.f;
  if (out64) {
    out64->vd = (va - vb) * f;
    out64->vb = vb * f;
    out64->sa = sa * f;
    out64->sb = sb * f;
    out64->pa = pa * f;
    out64->pb = pb * f;
    out64->td = (ta - tb) * f;
    out64->tb = tb * f;
    out64->da = da * f;
    for (int m = 0; m < 8; ++m) out64->m[m] = 0.0;
  }
  if (M576) {
    std::vector<double> Mm;
    to_modal(M576, Mm);
    double mmax = 0, mdev = 0;
    for (int i = 0; i < 576; ++i) mmax = std::max(mmax, std::fabs(Mm[i]));
    for (int i = 0; i < 24; ++i)
      for (int j = 0; j < 24; ++j) {
        const double expect = (i == j) ? Mm[(3 * (i / 3)) * 24 + 3 * (i / 3)] : 0.0;
        mdev = std::max(mdev, std::fabs(Mm[i * 24 + j] - expect));
      }
    if (!(mdev <= 1e-11 * mmax))
      return set_error(ctx, MSG_ERR_NOT_STRUCTURED, "element mass lacks the cube's modal structure (%g)", mdev / mmax);
    for (int m = 0; m < 8; ++m) out->m[m] = (float)(Mm[(3 * m) * 24 + 3 * m] * cM / 64.0);
    if (out64)
      for (int m = 0; m < 8; ++m) out64->m[m] = Mm[(3 * m) * 24 + 3 * m] * cM / 64.0;
  }
  return MSG_OK;
}

// A context workspace buffer seen through the DevMem-style accessor.
struct WSlot {
  void* ptr = nullptr;
  template <class T> T* as() const { return static_cast<T*>(ptr); }
};

// Where a batch runs: stream, timing events, pinned flag words and the cached
// inner-loop graph (the context's own, or a serving lane's).
struct BlockExec {
  cudaStream_t st = nullptr;
  cudaEvent_t* ev = nullptr;      // 12 events
  int* h_flags = nullptr;         // pinned, >= 64 bytes
  int* d_hflags = nullptr;        // device address of h_flags when it is mapped (else null)
  cudaGraphExec_t* graph = nullptr;
  size_t* graph_key = nullptr;
  bool ctx_stats = true;          // accumulate the context's phase timings and launch samples
  // persistent grids (one CTA per SM walking the work items) or one CTA per
  // item, which lets the block scheduler interleave other streams' kernels
  // (higher-priority serving lanes) between items
  bool persistent = true;
};

// Everything one batch of solves on a structured lattice shares: sizes,
// operator coefficients (A = cK E Khat + cM Mhat), workspace, tensor maps.
// One coarse level (l >= 1) of the multigrid preconditioner: its lattice,
// operator coefficients (Khat scales with the element size 2^l h, the mass with
// its cube), maps, vectors b (restricted residual), x (iterate) and t (residual
// or smoothed iterate), the coarsened element field and its Jacobi diagonal.
struct GmgLevel {
  Lattice L;
  int nx = 0, ny = 0, nz = 0;  // elements per axis
  ModalC MC;
  double kdiag = 0.0, mdiag = 0.0;
  const int* interior = nullptr;
  const uint8_t* mask = nullptr;
  float *b = nullptr, *x = nullptr, *t = nullptr, *E32 = nullptr, *dinv = nullptr;
  int tiles_j = 0, n_tiles = 0, n_items = 0, grid = 0;
  CUtensorMap tm_x, tm_t, tm_e;
  size_t sweep_smem = 0;  // coarsest level: all sweeps in one k_coarse_sweeps launch (0: launch per sweep)
  // packed operator (k_lvl_op2) on this level: x patches, element patches, own b and dinv
  ModalCT<float2> MC2;
  int tiles_j2 = 0, n_tiles2 = 0, n_items2 = 0, grid2 = 0;
  CUtensorMap tm2_x, tm2_e, tm2_bo, tm2_dinvo;
};

struct BlockSys {
  BlockExec X;
  DevMem* own = nullptr;  // kWorkSlots buffers owned by a serving lane; nullptr: the context's workspace slots
  bool fixed = false;     // true-residual step after every graph chunk (batch-invariant trajectories)
  Lattice L;
  int R = 0, Rp = 0;
  size_t npad = 0, nvec = 0;
  int n_tiles = 0, tiles_jm = 0, n_tiles_m = 0, n_items_m = 0, grid_m = 0, n_upd = 0, n_bsq = 0;
  bool modal = true, mass = false;
  double cK = 1.0, cM = 0.0, kdiag = 0.0, mdiag = 0.0;
  KhatD KD;               // cK-scaled classes
  MassClasses<double> MD; // cM-scaled mass classes
  ModalC MC;
  const int* interior = nullptr;
  const uint8_t* mask = nullptr;
  WSlot x, r32, p, q, d, dinv, blat, E64, E32, part_op, part_up, scal, pB, rB, qB;
  size_t scal_bytes = 0;
  Scal s;
  int slot_alloc(Context* ctx, int slot, size_t bytes, void** out) {
    if (!own) return workspace(ctx, slot, bytes, out);
    if (own[slot].bytes < bytes) {
      own[slot].release();
      MSG_TRY(own[slot].alloc(ctx, bytes));
    }
    *out = own[slot].ptr;
    return MSG_OK;
  }
  CUtensorMap tm_rAm, tm_rBm, tm_qAm, tm_qBm, tm_pAm, tm_pBm, tm_dinvm, tm_em, tm_dm;
  // FP64 Walsh-mode true-residual step (modal loops): the iterate alternates
  // between x and xB (the step writes x + d + alpha p into the other buffer)
  WSlot xB;
  ModalCD MCD;
  int tiles_jr = 0, n_tiles_r = 0, n_items_r = 0, grid_r = 0;
  CUtensorMap tm_xr, tm_xBr, tm_dr, tm_pr, tm_er;
  // multigrid preconditioner: levels 1..n_lvl-1 (level 0 is this lattice), the
  // level-0 pre-smoothed iterate xs, the damping and the coarsest-level sweeps
  bool gmg = false;
  int n_lvl = 1, sweeps = 0;
  float omega = 0.f;
  GmgLevel lv[kGmgMaxLevels];
  WSlot xs, arena;
  CUtensorMap tm_xs;
  // packed level-0 operator (k_lvl_op2: 64 realizations per item, 3 x 3 tiles)
  bool pack = false;
  ModalCT<float2> MC2;
  int tiles_j2 = 0, n_tiles2 = 0, n_items2 = 0, grid2 = 0;
  CUtensorMap tm2_rA, tm2_rB, tm2_qA, tm2_qB, tm2_pA, tm2_pB, tm2_xs, tm2_dinv, tm2_e, tm2_d;
  CUtensorMap tm2_rAo, tm2_rBo, tm2_dinvo;  // own-tile boxes of r (both buffers) and dinv (post-sweep)
  // level-0 search-direction launch on the tensor cores (k_lvl_tc): the B operand
  // image of cK Khat (4 corner pairs x [hi | lo] x 8 slots, K-major core matrices)
  bool tc = false;
  WSlot tc_bops;
};

// B operands of k_lvl_tc from the unit-cube element matrix: for corner pair
// (ax, ay) = pr, row n < 32 holds the TF32 high part and row 32 + n the low
// part of output column n = ((ax' 2 + ay') 2 + az') 3 + c' (n < 24; rows 24..31
// zero), slot k = az 3 + c (k < 6; slots 6, 7 zero) of cK Khat; K-major core
// matrices of 8 rows x 4 slots (LBO 128 B between the slot halves, SBO 256 B
// between 8-row groups), 2 KB per pair. Uploaded into workspace slot 33.
static int tc_setup(Context* ctx, BlockSys* B, const double* K576) {
  std::vector<float> img(kTcBFloats, 0.f);
  auto trunc_tf32 = [](float x) {
    uint32_t u;
    std::memcpy(&u, &x, 4);
    u &= 0xffffe000u;
    float y;
    std::memcpy(&y, &u, 4);
    return y;
  };
  for (int pr = 0; pr < 4; ++pr) {
    const int ax = pr >> 1, ay = pr & 1;
    for (int n = 0; n < 24; ++n) {
      const int c2 = n % 3, az2 = (n / 3) & 1, ay2 = (n / 6) & 1, ax2 = n / 12;
      const int row = corner_id(ax2, ay2, az2) * 3 + c2;
      for (int k = 0; k < 6; ++k) {
        const int az = k / 3, c = k % 3;
        const float f = (float)(B->cK * K576[row * 24 + corner_id(ax, ay, az) * 3 + c]);
        const float hi = trunc_tf32(f), lo = f - hi;
        for (int h = 0; h < 2; ++h) {
          const int nn = n + 32 * h;
          img[pr * 512 + (nn / 8) * 64 + (k / 4) * 32 + (nn % 8) * 4 + (k % 4)] = h ? lo : hi;
        }
      }
    }
  }
  MSG_TRY(B->slot_alloc(ctx, 33, sizeof(float) * img.size(), &B->tc_bops.ptr));
  MSG_CUDA(ctx, cudaMemcpyAsync(B->tc_bops.ptr, img.data(), sizeof(float) * img.size(), cudaMemcpyHostToDevice,
                                B->X.st));
  MSG_CUDA(ctx, cudaStreamSynchronize(B->X.st));
  static std::once_flag once;
  static cudaError_t attr = cudaSuccess;
  std::call_once(once, [] {
    attr = cudaFuncSetAttribute(k_lvl_tc<kLvlPcgZ>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTcSmem);
  });
  MSG_CUDA(ctx, attr);
  return MSG_OK;
}

// Largest eigenvalue of diag(K)^-1 K for one element (power iteration on the
// symmetric D^-1/2 K D^-1/2 from a fixed vector with no rigid-body part). It
// bounds the spectrum of the assembled Jacobi-scaled operator for any positive
// element field, so it fixes a safe Jacobi damping for every level.
double element_jacobi_lambda(const double* K576) {
  double dh[24], v[24], w[24];
  for (int i = 0; i < 24; ++i) {
    dh[i] = 1.0 / std::sqrt(K576[i * 24 + i]);
    v[i] = std::sin(1.7 * i + 0.3) + 0.01 * i;
  }
  double lam = 0.0;
  for (int it = 0; it < 500; ++it) {
    double nv = 0.0;
    for (int i = 0; i < 24; ++i) nv += v[i] * v[i];
    nv = std::sqrt(nv);
    for (int i = 0; i < 24; ++i) v[i] /= nv;
    for (int i = 0; i < 24; ++i) {
      double a = 0.0;
      for (int j = 0; j < 24; ++j) a += dh[i] * K576[i * 24 + j] * dh[j] * v[j];
      w[i] = a;
    }
    lam = 0.0;
    for (int i = 0; i < 24; ++i) lam += v[i] * w[i];
    for (int i = 0; i < 24; ++i) v[i] = w[i];
  }
  return lam;
}

// Coarse-level maps of a structured mesh for levels 1..n_lvl-1 (built once per
// mesh, under its lock): a coarse node is constrained in component c when the
// fine node it sits on is.
int gmg_maps(Context* ctx, Mesh* m, int n_lvl) {
  std::lock_guard<std::mutex> lock(m->gmg_mu);
  if (m->gmg_levels >= n_lvl) return MSG_OK;
  const int NXf = m->nx + 1, NYf = m->ny + 1;
  for (int l = m->gmg_levels; l < n_lvl; ++l) {
    const int nx = m->nx >> l, ny = m->ny >> l, nz = m->nz >> l;
    const int NX = nx + 1, NY = ny + 1, NZ = nz + 1, NXp = NX + 2, NYp = NY + 2, NZp = NZ + 2;
    std::vector<uint8_t> mask((size_t)NXp * NYp * NZp, 7);
    std::vector<int> interior((size_t)NX * NY * NZ);
    size_t t = 0;
    for (int k = 0; k < NZ; ++k)
      for (int j = 0; j < NY; ++j)
        for (int i = 0; i < NX; ++i, ++t) {
          const int p = (i + 1) + NXp * ((j + 1) + NYp * (k + 1));
          const size_t f = ((size_t)i << l) + (size_t)NXf * (((size_t)j << l) + (size_t)NYf * ((size_t)k << l));
          uint8_t mk = 0;
          for (int c = 0; c < 3; ++c)
            if (m->dof[3 * f + c] < 0) mk |= (uint8_t)(1 << c);
          mask[p] = mk;
          interior[t] = p;
        }
    MSG_TRY(m->d_gmg_mask[l].alloc(ctx, mask.size()));
    MSG_TRY(m->d_gmg_interior[l].alloc(ctx, sizeof(int) * interior.size()));
    MSG_CUDA(ctx, cudaMemcpy(m->d_gmg_mask[l].ptr, mask.data(), mask.size(), cudaMemcpyHostToDevice));
    MSG_CUDA(ctx, cudaMemcpy(m->d_gmg_interior[l].ptr, interior.data(), sizeof(int) * interior.size(),
                             cudaMemcpyHostToDevice));
  }
  m->gmg_levels = n_lvl;
  return MSG_OK;
}

// Coefficients and workspace of a batch: A = cK E Khat(nu) + cM Mhat(rho).
int block_setup(Context* ctx, Mesh* m, double nu, double rho, double cK, double cM, int R, int Rp, BlockSys* B,
                DevMem* own = nullptr, const BlockExec* exec = nullptr) {
  if (!m->structured) return set_error(ctx, MSG_ERR_NOT_STRUCTURED, "mesh is not a structured cube lattice");
  B->own = own;
  if (exec) {
    B->X = *exec;
  } else {
    MSG_TRY(context_resources(ctx));
    B->X.st = ctx->stream;
    B->X.ev = ctx->ev;
    B->X.h_flags = ctx->h_flags;
    B->X.d_hflags = ctx->d_hflags;
    B->X.graph = &ctx->batch_graph;
    B->X.graph_key = &ctx->batch_graph_key;
    B->X.ctx_stats = true;
  }
  Lattice& L = B->L;
  L.NX = m->nx + 1; L.NY = m->ny + 1; L.NZ = m->nz + 1;
  L.NXp = m->NXp; L.NYp = m->NYp; L.NZp = m->NZp;
  L.Rp = Rp;
  L.tiles_j = (L.NY + kTJ - 1) / kTJ;
  L.n_pad = L.NXp * L.NYp * L.NZp;
  L.n_int = L.NX * L.NY * L.NZ;
  B->R = R;
  B->Rp = Rp;
  B->n_tiles = L.tiles_j * ((L.NZ + kTK - 1) / kTK);
  B->npad = (size_t)L.n_pad;
  B->nvec = B->npad * 3 * Rp;
  B->interior = m->d_pad_interior.as<int>();
  B->mask = m->d_pad_mask.as<uint8_t>();
  B->cK = cK;
  B->cM = cM;
  B->mass = cM != 0.0;
  B->modal = true;  // the Walsh-mode operator (every batched loop)
  cudaStream_t st = B->X.st;

  double K576[576];
  MSG_TRY(unit_cube_khat(ctx, m->h, nu, K576));
  for (int c = 0; c < kKhatClasses; ++c) {
    const double v = K576[kKhatRep[c]];
    B->KD.v[c] = cK * v;
  }
  for (int i = 0; i < 576; ++i) {  // the element must have the cube's class structure
    const int code = kKhatClass[i];
    const double v = code > 0 ? K576[kKhatRep[code - 1]] : -K576[kKhatRep[-code - 1]];
    if (std::fabs(v - K576[i]) > 1e-12 * std::fabs(K576[kKhatRep[0]]))
      return set_error(ctx, MSG_ERR_NOT_STRUCTURED, "element stiffness does not have the unit-cube structure");
  }
  B->kdiag = cK * K576[0];
  double M576[576];
  for (int i = 0; i < 4; ++i) B->MD.v[i] = 0.0;
  if (B->mass) {
    MSG_TRY(unit_cube_mhat(ctx, m->h, rho, M576));
    // classes by the number of differing corner coordinates; check the structure
    auto cc = [](int a, int k) {
      const int ax = (a == 1 || a == 2 || a == 5 || a == 6), ay = (a == 2 || a == 3 || a == 6 || a == 7), az = a >= 4;
      return k == 0 ? ax : (k == 1 ? ay : az);
    };
    auto dist = [&](int a, int b) { return (cc(a, 0) != cc(b, 0)) + (cc(a, 1) != cc(b, 1)) + (cc(a, 2) != cc(b, 2)); };
    double rep[4] = {0, 0, 0, 0};
    for (int b = 0; b < 8; ++b) rep[dist(0, b)] = M576[(3 * 0) * 24 + 3 * b];
    for (int a = 0; a < 8; ++a)
      for (int b = 0; b < 8; ++b)
        for (int c = 0; c < 3; ++c)
          for (int c2 = 0; c2 < 3; ++c2) {
            const double expect = c == c2 ? rep[dist(a, b)] : 0.0;
            if (std::fabs(M576[(3 * a + c) * 24 + 3 * b + c2] - expect) > 1e-12 * std::fabs(rep[0]))
              return set_error(ctx, MSG_ERR_NOT_STRUCTURED, "element mass does not have the cube structure");
          }
    for (int i = 0; i < 4; ++i) B->MD.v[i] = cM * rep[i];
    B->mdiag = cM * rep[0];
  }
  if (B->modal) MSG_TRY(modal_coefficients(ctx, K576, B->mass ? M576 : nullptr, cK, cM, &B->MC, &B->MCD));
  B->tiles_jm = (L.NY + kMJ - 1) / kMJ;
  B->n_tiles_m = B->tiles_jm * ((L.NZ + kMK - 1) / kMK);
  B->n_items_m = B->n_tiles_m * (Rp / 32);
  B->grid_m = B->X.persistent ? std::min(B->n_items_m, ctx->sm_count) : B->n_items_m;
  B->n_upd = std::min(L.n_int, ctx->sm_count * 4);
  B->n_bsq = std::min(L.n_int, ctx->sm_count * 2);

  // workspace (context slots, reused by the next batch)
  const size_t nvec = B->nvec, npad = B->npad;
  MSG_TRY(B->slot_alloc(ctx, 0, sizeof(double) * nvec, &B->x.ptr));
  MSG_TRY(B->slot_alloc(ctx, 1, sizeof(float) * nvec, &B->r32.ptr));
  MSG_TRY(B->slot_alloc(ctx, 2, sizeof(float) * nvec, &B->p.ptr));
  MSG_TRY(B->slot_alloc(ctx, 3, sizeof(float) * nvec, &B->q.ptr));
  MSG_TRY(B->slot_alloc(ctx, 4, sizeof(float) * nvec, &B->d.ptr));
  MSG_TRY(B->slot_alloc(ctx, 5, sizeof(float) * npad * Rp, &B->dinv.ptr));
  MSG_TRY(B->slot_alloc(ctx, 6, sizeof(double) * npad * Rp, &B->E64.ptr));
  MSG_TRY(B->slot_alloc(ctx, 7, sizeof(float) * npad * Rp, &B->E32.ptr));
  MSG_TRY(B->slot_alloc(ctx, 8, sizeof(double) * npad * 3, &B->blat.ptr));
  MSG_TRY(B->slot_alloc(ctx, 9, sizeof(double) * (size_t)std::max(B->n_tiles * 2, B->n_tiles_m * kMParts) * Rp,
                    &B->part_op.ptr));
  MSG_TRY(B->slot_alloc(ctx, 10, sizeof(double) * (size_t)std::max(B->n_upd, B->n_bsq) * Rp * 2, &B->part_up.ptr));
  B->scal_bytes = (sizeof(float) * 2 + sizeof(double) * 6 + sizeof(int) * 5) * (size_t)Rp + 64;
  MSG_TRY(B->slot_alloc(ctx, 11, B->scal_bytes, &B->scal.ptr));
  if (B->modal) {  // second buffers of p, r and q for the single-reduction loop, and of x
    MSG_TRY(B->slot_alloc(ctx, 18, sizeof(float) * nvec, &B->pB.ptr));
    MSG_TRY(B->slot_alloc(ctx, 19, sizeof(float) * nvec, &B->rB.ptr));
    MSG_TRY(B->slot_alloc(ctx, 20, sizeof(float) * nvec, &B->qB.ptr));
    MSG_TRY(B->slot_alloc(ctx, 32, sizeof(double) * nvec, &B->xB.ptr));
    MSG_CUDA(ctx, cudaMemsetAsync(B->xB.ptr, 0, sizeof(double) * nvec, st));
  }
  Scal& sc = B->s;
  {
    char* base = B->scal.as<char>();
    sc.alpha = (float*)base; base += sizeof(float) * Rp;
    sc.beta = (float*)base; base += sizeof(float) * Rp;
    sc.gamma = (double*)base; base += sizeof(double) * Rp;
    sc.gamma_prev = (double*)base; base += sizeof(double) * Rp;
    sc.rho_ref = (double*)base; base += sizeof(double) * Rp;
    sc.res = (double*)base; base += sizeof(double) * Rp;
    sc.bnorm = (double*)base; base += sizeof(double) * Rp;
    sc.gamma0 = (double*)base; base += sizeof(double) * Rp;
    sc.act = (int*)base; base += sizeof(int) * Rp;
    sc.done = (int*)base; base += sizeof(int) * Rp;
    sc.its = (int*)base; base += sizeof(int) * Rp;
    sc.breakdown = (int*)base; base += sizeof(int) * Rp;
    sc.fresh = (int*)base; base += sizeof(int) * Rp;
    sc.n_active = (int*)base; base += 16;
    sc.n_update = (int*)base; base += 16;
    sc.err = (int*)base;  // outside the 32 bytes the iterations clear
  }
  // zero every padded vector once: ghost entries must stay zero
  const WSlot* v32[] = {&B->r32, &B->p, &B->q, &B->d, &B->pB, &B->rB, &B->qB};
  for (const WSlot* w : v32)
    if (w->ptr) MSG_CUDA(ctx, cudaMemsetAsync(w->ptr, 0, sizeof(float) * nvec, st));
  MSG_CUDA(ctx, cudaMemsetAsync(B->x.ptr, 0, sizeof(double) * nvec, st));
  MSG_CUDA(ctx, cudaMemsetAsync(B->dinv.ptr, 0, sizeof(float) * npad * Rp, st));
  MSG_CUDA(ctx, cudaMemsetAsync(B->E64.ptr, 0, sizeof(double) * npad * Rp, st));
  MSG_CUDA(ctx, cudaMemsetAsync(B->E32.ptr, 0, sizeof(float) * npad * Rp, st));  // ghost elements stay 0
  MSG_CUDA(ctx, cudaMemsetAsync(B->blat.ptr, 0, sizeof(double) * npad * 3, st));

  // TMA descriptors of the FP32 batch vectors (5-D: realization, component,
  // x, y, z) and of the FP32 element field and dinv (4-D: realization, x, y, z)
  static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult qr;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &qr) == cudaSuccess &&
        qr == cudaDriverEntryPointSuccess)
      encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
  });
  if (!encode) return set_error(ctx, MSG_ERR_CUDA, "cuTensorMapEncodeTiled is not available");
  const cuuint64_t fb = sizeof(float);
  const cuuint64_t pd[5] = {(cuuint64_t)Rp, 3, (cuuint64_t)L.NXp, (cuuint64_t)L.NYp, (cuuint64_t)L.NZp};
  const cuuint64_t ps[4] = {Rp * fb, 3 * Rp * fb, 3 * Rp * fb * L.NXp, 3 * Rp * fb * L.NXp * L.NYp};
  const cuuint64_t ed[4] = {(cuuint64_t)Rp, (cuuint64_t)L.NXp, (cuuint64_t)L.NYp, (cuuint64_t)L.NZp};
  const cuuint64_t es[3] = {Rp * fb, Rp * fb * L.NXp, Rp * fb * L.NXp * L.NYp};
  const cuuint32_t one[5] = {1, 1, 1, 1, 1};
  auto enc5 = [&](CUtensorMap* tm, void* base, const cuuint32_t* box) {
    return encode(tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 5, base, pd, ps, box, one, CU_TENSOR_MAP_INTERLEAVE_NONE,
                  CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  };
  auto enc4 = [&](CUtensorMap* tm, void* base, const cuuint32_t* box) {
    return encode(tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, base, ed, es, box, one, CU_TENSOR_MAP_INTERLEAVE_NONE,
                  CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  };
  CUresult e = CUDA_SUCCESS;
  if (B->modal) {
    // modal loop: r, q, p (both buffers) and dinv patches with halo, the element patch, the tile's d
    const cuuint32_t pbm[5] = {32, 3, 1, kMPJ, kMPK};
    const cuuint32_t nbm[4] = {32, 1, kMPJ, kMPK};
    const cuuint32_t ebm[4] = {32, 1, kMEJ, kMEK};
    const cuuint32_t dbm[5] = {32, 3, 1, kMJ, kMK};
    const CUresult rs[9] = {enc5(&B->tm_rAm, B->r32.ptr, pbm), enc5(&B->tm_rBm, B->rB.ptr, pbm),
                            enc5(&B->tm_qAm, B->q.ptr, pbm),   enc5(&B->tm_qBm, B->qB.ptr, pbm),
                            enc5(&B->tm_pAm, B->p.ptr, pbm),   enc5(&B->tm_pBm, B->pB.ptr, pbm),
                            enc4(&B->tm_dinvm, B->dinv.ptr, nbm), enc4(&B->tm_em, B->E32.ptr, ebm),
                            enc5(&B->tm_dm, B->d.ptr, dbm)};
    for (CUresult r : rs)
      if (r != CUDA_SUCCESS) e = r;
    // FP64 true-residual step: x (both buffers, FP64), d and p (FP32) patches
    // of a 3 x 2 node tile with halo, the FP64 element patch
    {
      const cuuint64_t db = sizeof(double);
      const cuuint64_t ps64[4] = {Rp * db, 3 * Rp * db, 3 * Rp * db * L.NXp, 3 * Rp * db * L.NXp * L.NYp};
      const cuuint64_t es64[3] = {Rp * db, Rp * db * L.NXp, Rp * db * L.NXp * L.NYp};
      const cuuint32_t rbox[5] = {32, 3, 1, kRPJ, kRPK};
      const cuuint32_t rebox[4] = {32, 1, kREJ, kREK};
      auto enc64 = [&](CUtensorMap* tm, void* base) {
        return encode(tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 5, base, pd, ps64, rbox, one, CU_TENSOR_MAP_INTERLEAVE_NONE,
                      CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                      CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
      };
      const CUresult r64[5] = {
          enc64(&B->tm_xr, B->x.ptr), enc64(&B->tm_xBr, B->xB.ptr), enc5(&B->tm_dr, B->d.ptr, rbox),
          enc5(&B->tm_pr, B->p.ptr, rbox),
          encode(&B->tm_er, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, B->E64.ptr, ed, es64, rebox, one,
                 CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                 CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE)};
      for (CUresult r : r64)
        if (r != CUDA_SUCCESS) e = r;
      B->tiles_jr = (L.NY + kRJ - 1) / kRJ;
      B->n_tiles_r = B->tiles_jr * ((L.NZ + kRK - 1) / kRK);
      B->n_items_r = B->n_tiles_r * (Rp / 32);
      B->grid_r = B->X.persistent ? std::min(B->n_items_r, ctx->sm_count) : B->n_items_r;
    }
    static std::once_flag resid_once;
    static cudaError_t resid_err = cudaSuccess;
    std::call_once(resid_once, [] {
      const void* fs[] = {(const void*)k_resid_modal<false, false, false>, (const void*)k_resid_modal<false, false, true>,
                          (const void*)k_resid_modal<false, true, false>,  (const void*)k_resid_modal<false, true, true>,
                          (const void*)k_resid_modal<true, false, false>,  (const void*)k_resid_modal<true, false, true>,
                          (const void*)k_resid_modal<true, true, false>,   (const void*)k_resid_modal<true, true, true>};
      for (const void* f : fs)
        if (resid_err == cudaSuccess)
          resid_err = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kRSmem);
    });
    MSG_CUDA(ctx, resid_err);
    static std::once_flag attr_once;
    static cudaError_t attr_err = cudaSuccess;
    std::call_once(attr_once, [] {
      attr_err = cudaFuncSetAttribute(k_op_modal<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kMSmem);
      if (attr_err == cudaSuccess)
        attr_err = cudaFuncSetAttribute(k_op_modal<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kMSmem);
    });
    MSG_CUDA(ctx, attr_err);
  }
  if (e != CUDA_SUCCESS) return set_error(ctx, MSG_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)e);

  // multigrid levels: halve the lattice while every axis is even and keeps at
  // least 2 elements
  B->gmg = false;
  B->n_lvl = 1;
  // (by default only without a mass term: a mass-dominated system, as in implicit
  // dynamics, is close to diagonal and the Jacobi loop needs few cheaper iterations)
  if (B->modal && (ctx->multigrid == 2 || (ctx->multigrid == 1 && !B->mass))) {
    int n_lvl = 1;
    while (n_lvl < ctx->mg_levels) {
      const int nx = m->nx >> (n_lvl - 1), ny = m->ny >> (n_lvl - 1), nz = m->nz >> (n_lvl - 1);
      if ((nx & 1) || (ny & 1) || (nz & 1) || nx < 4 || ny < 4 || nz < 4) break;
      ++n_lvl;
    }
    if (n_lvl >= 2) {
      MSG_TRY(gmg_maps(ctx, m, n_lvl));
      B->gmg = true;
      B->n_lvl = n_lvl;
      B->sweeps = ctx->mg_sweeps;
      const double lam = element_jacobi_lambda(K576);
      B->omega = (float)(ctx->mg_omega > 0.0 ? ctx->mg_omega : std::min(0.6, 3.19 / lam));
      MSG_TRY(B->slot_alloc(ctx, 30, sizeof(float) * nvec, &B->xs.ptr));
      MSG_CUDA(ctx, cudaMemsetAsync(B->xs.ptr, 0, sizeof(float) * nvec, st));
      const cuuint32_t pbm[5] = {32, 3, 1, kMPJ, kMPK};
      if (enc5(&B->tm_xs, B->xs.ptr, pbm) != CUDA_SUCCESS)
        return set_error(ctx, MSG_ERR_CUDA, "cuTensorMapEncodeTiled failed (multigrid)");
      size_t arena = 0;
      auto take = [&](size_t bytes) {
        const size_t o = arena;
        arena += (bytes + 255) & ~(size_t)255;
        return o;
      };
      size_t off[kGmgMaxLevels][5];
      for (int l = 1; l < n_lvl; ++l) {
        GmgLevel& g = B->lv[l];
        g.nx = m->nx >> l;
        g.ny = m->ny >> l;
        g.nz = m->nz >> l;
        Lattice& Lc = g.L;
        Lc.NX = g.nx + 1; Lc.NY = g.ny + 1; Lc.NZ = g.nz + 1;
        Lc.NXp = Lc.NX + 2; Lc.NYp = Lc.NY + 2; Lc.NZp = Lc.NZ + 2;
        Lc.Rp = Rp;
        Lc.tiles_j = (Lc.NY + kTJ - 1) / kTJ;
        Lc.n_pad = Lc.NXp * Lc.NYp * Lc.NZp;
        Lc.n_int = Lc.NX * Lc.NY * Lc.NZ;
        const double sk = (double)(1 << l), sm = sk * sk * sk;
        MSG_TRY(modal_coefficients(ctx, K576, B->mass ? M576 : nullptr, cK * sk, cM * sm, &g.MC));
        g.kdiag = B->kdiag * sk;
        g.mdiag = B->mdiag * sm;
        g.interior = m->d_gmg_interior[l].as<int>();
        g.mask = m->d_gmg_mask[l].as<uint8_t>();
        g.tiles_j = (Lc.NY + kMJ - 1) / kMJ;
        g.n_tiles = g.tiles_j * ((Lc.NZ + kMK - 1) / kMK);
        g.n_items = g.n_tiles * (Rp / 32);
        g.grid = B->X.persistent ? std::min(g.n_items, ctx->sm_count) : g.n_items;
        const size_t nv = (size_t)Lc.n_pad * 3 * Rp, ns = (size_t)Lc.n_pad * Rp;
        off[l][0] = take(sizeof(float) * nv);
        off[l][1] = take(sizeof(float) * nv);
        off[l][2] = take(sizeof(float) * nv);
        off[l][3] = take(sizeof(float) * ns);
        off[l][4] = take(sizeof(float) * ns);
      }
      MSG_TRY(B->slot_alloc(ctx, 31, arena, &B->arena.ptr));
      MSG_CUDA(ctx, cudaMemsetAsync(B->arena.ptr, 0, arena, st));  // ghosts stay zero
      char* base = B->arena.as<char>();
      for (int l = 1; l < n_lvl; ++l) {
        GmgLevel& g = B->lv[l];
        g.b = (float*)(base + off[l][0]);
        g.x = (float*)(base + off[l][1]);
        g.t = (float*)(base + off[l][2]);
        g.E32 = (float*)(base + off[l][3]);
        g.dinv = (float*)(base + off[l][4]);
        const Lattice& Lc = g.L;
        const cuuint64_t cpd[5] = {(cuuint64_t)Rp, 3, (cuuint64_t)Lc.NXp, (cuuint64_t)Lc.NYp, (cuuint64_t)Lc.NZp};
        const cuuint64_t cps[4] = {Rp * fb, 3 * Rp * fb, 3 * Rp * fb * Lc.NXp, 3 * Rp * fb * Lc.NXp * Lc.NYp};
        const cuuint64_t ced[4] = {(cuuint64_t)Rp, (cuuint64_t)Lc.NXp, (cuuint64_t)Lc.NYp, (cuuint64_t)Lc.NZp};
        const cuuint64_t ces[3] = {Rp * fb, Rp * fb * Lc.NXp, Rp * fb * Lc.NXp * Lc.NYp};
        const cuuint32_t ebm[4] = {32, 1, kMEJ, kMEK};
        auto c5 = [&](CUtensorMap* tm, void* p) {
          return encode(tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 5, p, cpd, cps, pbm, one, CU_TENSOR_MAP_INTERLEAVE_NONE,
                        CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        };
        const CUresult r1 = c5(&g.tm_x, g.x), r2 = c5(&g.tm_t, g.t);
        const CUresult r3 = encode(&g.tm_e, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, g.E32, ced, ces, ebm, one,
                                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                   CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r1 != CUDA_SUCCESS || r2 != CUDA_SUCCESS || r3 != CUDA_SUCCESS)
          return set_error(ctx, MSG_ERR_CUDA, "cuTensorMapEncodeTiled failed (multigrid level %d)", l);
      }
      {  // coarsest level: one launch for all its sweeps when it fits a CTA
        GmgLevel& g = B->lv[n_lvl - 1];
        const size_t sm = coarse_sweep_smem(g.L);
        g.sweep_smem = (ctx->mg_fused_coarse && g.L.NY <= kMJ && g.L.NZ <= kMK && sm <= 200 * 1024) ? sm : 0;
        if (g.sweep_smem) {
          static std::once_flag cs_once;
          static cudaError_t cs_err = cudaSuccess;
          std::call_once(cs_once, [] {
            cs_err = cudaFuncSetAttribute(k_coarse_sweeps<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          200 * 1024);
            if (cs_err == cudaSuccess)
              cs_err = cudaFuncSetAttribute(k_coarse_sweeps<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            200 * 1024);
          });
          MSG_CUDA(ctx, cs_err);
        }
      }
      // level-0 search direction on the tensor cores (no mass term)
      B->tc = ctx->tensor_op != 0 && !B->mass;
      if (B->tc) MSG_TRY(tc_setup(ctx, B, K576));
      // packed level-0 operator: realizations in multiples of 64
      B->pack = ctx->mg_packed && (Rp % kQR) == 0;
      if (B->pack) {
        auto b2 = [](float v) { return make_float2(v, v); };
        auto pack_c = [&](const ModalC& f, ModalCT<float2>& g2) {
          g2.vd = b2(f.vd); g2.vb = b2(f.vb); g2.sa = b2(f.sa); g2.sb = b2(f.sb); g2.pa = b2(f.pa); g2.pb = b2(f.pb);
          g2.td = b2(f.td); g2.tb = b2(f.tb); g2.da = b2(f.da);
          for (int i = 0; i < 8; ++i) g2.m[i] = b2(f.m[i]);
        };
        pack_c(B->MC, B->MC2);
        B->tiles_j2 = (L.NY + kQJ - 1) / kQJ;
        B->n_tiles2 = B->tiles_j2 * ((L.NZ + kQK - 1) / kQK);
        B->n_items2 = B->n_tiles2 * (Rp / kQR);
        B->grid2 = B->X.persistent ? std::min(B->n_items2, ctx->sm_count) : B->n_items2;
        // the loop's partials: [tile][Rp][2] and [tile][Rp] over the packed tiles
        const size_t need = sizeof(double) * (size_t)std::max({B->n_tiles * 2, B->n_tiles_m * kMParts,
                                                                B->n_tiles2 * 3}) * Rp;
        MSG_TRY(B->slot_alloc(ctx, 9, need, &B->part_op.ptr));
        const cuuint32_t pb2[5] = {kQR, 3, 1, kQPJ, kQPK};
        const cuuint32_t nb2[4] = {kQR, 1, kQPJ, kQPK};
        const cuuint32_t eb2[4] = {kQR, 1, kQEJ, kQEK};
        const cuuint32_t db2[5] = {kQR, 3, 1, kQJ, kQK};
        const cuuint32_t ob2[4] = {kQR, 1, kQJ, kQK};
        if (enc5(&B->tm2_rAo, B->r32.ptr, db2) != CUDA_SUCCESS || enc5(&B->tm2_rBo, B->rB.ptr, db2) != CUDA_SUCCESS ||
            enc4(&B->tm2_dinvo, B->dinv.ptr, ob2) != CUDA_SUCCESS)
          return set_error(ctx, MSG_ERR_CUDA, "cuTensorMapEncodeTiled failed (packed)");
        const CUresult r2[10] = {enc5(&B->tm2_rA, B->r32.ptr, pb2), enc5(&B->tm2_rB, B->rB.ptr, pb2),
                                 enc5(&B->tm2_qA, B->q.ptr, pb2),   enc5(&B->tm2_qB, B->qB.ptr, pb2),
                                 enc5(&B->tm2_pA, B->p.ptr, pb2),   enc5(&B->tm2_pB, B->pB.ptr, pb2),
                                 enc5(&B->tm2_xs, B->xs.ptr, pb2),  enc4(&B->tm2_dinv, B->dinv.ptr, nb2),
                                 enc4(&B->tm2_e, B->E32.ptr, eb2),  enc5(&B->tm2_d, B->d.ptr, db2)};
        for (CUresult r : r2)
          if (r != CUDA_SUCCESS) return set_error(ctx, MSG_ERR_CUDA, "cuTensorMapEncodeTiled failed (packed)");
        // the coarse levels' residual and post-sweeps on the packed operator too
        for (int l = 1; l < n_lvl; ++l) {
          GmgLevel& g = B->lv[l];
          const Lattice& Lc = g.L;
          pack_c(g.MC, g.MC2);
          g.tiles_j2 = (Lc.NY + kQJ - 1) / kQJ;
          g.n_tiles2 = g.tiles_j2 * ((Lc.NZ + kQK - 1) / kQK);
          g.n_items2 = g.n_tiles2 * (Rp / kQR);
          g.grid2 = B->X.persistent ? std::min(g.n_items2, ctx->sm_count) : g.n_items2;
          const cuuint64_t cpd[5] = {(cuuint64_t)Rp, 3, (cuuint64_t)Lc.NXp, (cuuint64_t)Lc.NYp, (cuuint64_t)Lc.NZp};
          const cuuint64_t cps[4] = {Rp * fb, 3 * Rp * fb, 3 * Rp * fb * Lc.NXp, 3 * Rp * fb * Lc.NXp * Lc.NYp};
          const cuuint64_t ced[4] = {(cuuint64_t)Rp, (cuuint64_t)Lc.NXp, (cuuint64_t)Lc.NYp, (cuuint64_t)Lc.NZp};
          const cuuint64_t ces[3] = {Rp * fb, Rp * fb * Lc.NXp, Rp * fb * Lc.NXp * Lc.NYp};
          auto l5 = [&](CUtensorMap* tm, void* p, const cuuint32_t* box) {
            return encode(tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 5, p, cpd, cps, box, one, CU_TENSOR_MAP_INTERLEAVE_NONE,
                          CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
          };
          auto l4 = [&](CUtensorMap* tm, void* p, const cuuint32_t* box) {
            return encode(tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, p, ced, ces, box, one, CU_TENSOR_MAP_INTERLEAVE_NONE,
                          CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
          };
          const CUresult rl[4] = {l5(&g.tm2_x, g.x, pb2), l4(&g.tm2_e, g.E32, eb2), l5(&g.tm2_bo, g.b, db2),
                                  l4(&g.tm2_dinvo, g.dinv, ob2)};
          for (CUresult r : rl)
            if (r != CUDA_SUCCESS)
              return set_error(ctx, MSG_ERR_CUDA, "cuTensorMapEncodeTiled failed (packed level %d)", l);
        }
        static std::once_flag pack_once;
        static cudaError_t pack_err = cudaSuccess;
        std::call_once(pack_once, [] {
          const std::pair<const void*, size_t> fs[] = {
              {(const void*)k_lvl_op2<kLvlResid, false>, LvlStage2<kLvlResid>::kSmem},
              {(const void*)k_lvl_op2<kLvlResid, true>, LvlStage2<kLvlResid>::kSmem},
              {(const void*)k_lvl_op2<kLvlStart, false>, LvlStage2<kLvlStart>::kSmem},
              {(const void*)k_lvl_op2<kLvlStart, true>, LvlStage2<kLvlStart>::kSmem},
              {(const void*)k_lvl_op2<kLvlSmooth, false>, LvlStage2<kLvlSmooth>::kSmem},
              {(const void*)k_lvl_op2<kLvlSmooth, true>, LvlStage2<kLvlSmooth>::kSmem},
              {(const void*)k_lvl_op2<kLvlPcgZ, false>, LvlStage2<kLvlPcgZ>::kSmem},
              {(const void*)k_lvl_op2<kLvlPcgZ, true>, LvlStage2<kLvlPcgZ>::kSmem}};
          for (const auto& f : fs)
            if (pack_err == cudaSuccess)
              pack_err = cudaFuncSetAttribute(f.first, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)f.second);
        });
        MSG_CUDA(ctx, pack_err);
      }
      static std::once_flag lvl_once;
      static cudaError_t lvl_err = cudaSuccess;
      std::call_once(lvl_once, [] {
        const std::pair<const void*, size_t> fs[] = {
            {(const void*)k_lvl_op<kLvlStart, false>, LvlStage<kLvlStart>::kSmem},
            {(const void*)k_lvl_op<kLvlStart, true>, LvlStage<kLvlStart>::kSmem},
            {(const void*)k_lvl_op<kLvlResid, false>, LvlStage<kLvlResid>::kSmem},
            {(const void*)k_lvl_op<kLvlResid, true>, LvlStage<kLvlResid>::kSmem},
            {(const void*)k_lvl_op<kLvlSmooth, false>, LvlStage<kLvlSmooth>::kSmem},
            {(const void*)k_lvl_op<kLvlSmooth, true>, LvlStage<kLvlSmooth>::kSmem},
            {(const void*)k_lvl_op<kLvlPcgZ, false>, LvlStage<kLvlPcgZ>::kSmem},
            {(const void*)k_lvl_op<kLvlPcgZ, true>, LvlStage<kLvlPcgZ>::kSmem}};
        for (const auto& f : fs)
          if (lvl_err == cudaSuccess)
            lvl_err = cudaFuncSetAttribute(f.first, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)f.second);
      });
      MSG_CUDA(ctx, lvl_err);
    }
  }
  return MSG_OK;
}

// Multigrid: coarsened element fields and the Jacobi diagonal of every coarse
// level, for all realizations (a realization whose fine field did not change
// gets the same values again).
void gmg_fields(Context* ctx, BlockSys* B, cudaStream_t st) {
  for (int l = 1; l < B->n_lvl; ++l) {
    GmgLevel& g = B->lv[l];
    const Lattice& Lf = l == 1 ? B->L : B->lv[l - 1].L;
    const float* Ef = l == 1 ? B->E32.as<float>() : B->lv[l - 1].E32;
    k_coarsen_E<<<g.nx * g.ny * g.nz, 128, 0, st>>>(Lf, g.L, g.nx, g.ny, Ef, g.E32);
    k_dinv<<<g.L.n_int, 128, 0, st>>>(g.L, g.kdiag, g.mdiag, g.E32, g.interior, g.dinv);
    count_launch(ctx, 2);
  }
}

// Field of every realization straight into the padded element layout (FP64
// and FP32), and the Jacobi diagonal of A.
int block_field(Context* ctx, Mesh* m, BlockSys* B, const KLDevice* kl, const double* d_xi) {
  cudaStream_t st = ctx->stream;
  MSG_TRY(context_resources(ctx));
  cudaEvent_t* ev = ctx->ev;
  cudaEventRecord(ev[10], st);
  MSG_TRY(launch_kl_field(ctx, m, kl, B->R, B->Rp, d_xi, B->E64.as<double>(), nullptr, nullptr,
                          m->d_pad_elem_row.as<int>()));
  k_f64_to_f32<<<ctx->sm_count * 8, 256, 0, st>>>(B->npad * B->Rp, B->E64.as<double>(), B->E32.as<float>());
  cudaEventRecord(ev[11], st);
  k_dinv<<<B->L.n_int, 128, 0, st>>>(B->L, B->kdiag, B->mdiag, B->E32.as<float>(), B->interior,
                                     B->dinv.as<float>());
  count_launch(ctx, 2);
  gmg_fields(ctx, B, st);
  MSG_CUDA(ctx, cudaGetLastError());
  return MSG_OK;
}

// Launch geometry and tolerances shared by the inner-loop graph and the
// true-residual step of a batch.
struct LoopCfg {
  int sblocks = 0, n_dir = 0, chunk = 2;
  double delta2 = 0.0, tol2 = 0.0;
};

LoopCfg loop_cfg(Context* ctx, const BlockSys* B, double tol, int chunk_cap) {
  LoopCfg c;
  const int Rp = B->Rp;
  c.sblocks = Rp / 32;  // scalar kernels: 32 realizations x 32 row groups per CTA
  c.n_dir = std::min(B->L.n_int, ctx->sm_count * 8);
  c.chunk = std::max(2, (chunk_cap > 0 ? std::min(ctx->chunk, chunk_cap) : ctx->chunk) & ~1);
  c.delta2 = ctx->reliable_delta * ctx->reliable_delta;
  if (B->gmg) {
    // a multigrid iteration cuts the residual several-fold: check every few
    // iterations, replace the residual after a larger drop
    c.chunk = 2;
    c.delta2 = ctx->mg_delta * ctx->mg_delta;
  }
  // ask for a check once sqrt(gamma / gamma0) is at tol/4 (single-reduction loop,
  // dinv-weighted norm), or once the recursive residual is at tol/2 (multigrid loop)
  c.tol2 = (!B->gmg ? 0.0625 : 0.25) * tol * tol;
  return c;
}

// One iteration of the multigrid-preconditioned loop (enqueued on st; every
// launch is a graph node while the chunk is captured). Level 0 (the batch
// lattice): r (r32 / rB alternating), the pre-smoothed iterate xs, the residual
// after pre-smoothing and later z (both in qB), p (p / pB alternating), q, d.
// V-cycle: one damped Jacobi sweep down (from zero), residual, restriction;
// `sweeps` sweeps on the coarsest level; prolongation and one sweep up. With
// the same sweep on both sides and a fixed sweep count on the coarsest level
// the preconditioner is symmetric positive definite (damping below
// 2 / lambda_max(dinv A)).
// The V-cycle of one iteration, from the level-0 start pass (r' = r - alpha q
// from r_in into r_out, pre-smoothing, residual) to the level-0 post-sweep
// (z into qB, partial z.r'), with the scalars of s.
void gmg_vcycle(BlockSys* B, Scal& s, bool even, cudaStream_t st) {
  const int Rp = B->Rp;
  const int nl = B->n_lvl;
  const float om = B->omega;
  double* part2 = B->part_op.as<double>();
  float* r_in = even ? B->r32.as<float>() : B->rB.as<float>();
  float* r_out = even ? B->rB.as<float>() : B->r32.as<float>();
  const CUtensorMap& tm_rin = even ? B->tm_rAm : B->tm_rBm;
  float* qB = B->qB.as<float>();
  const bool mass = B->mass;
  auto lvl = [&](auto mode, const Lattice& L, const ModalC& C, const CUtensorMap& ta, const CUtensorMap& tb,
                 const CUtensorMap& tn, const CUtensorMap& te, const CUtensorMap& td, int tiles_j, int n_tiles,
                 int n_items, int grid, const uint8_t* mask, const float* b, const float* dinv, float* out,
                 float* out2, float* out3, float* d, double* partial, int pstride) {
    constexpr int kMode = decltype(mode)::value;
    auto k = mass ? k_lvl_op<kMode, true> : k_lvl_op<kMode, false>;
    k<<<grid, kMThreads, LvlStage<kMode>::kSmem, st>>>(L, C, ta, tb, tn, te, td, tiles_j, n_tiles, n_items, mask, b,
                                                       dinv, om, s.alpha, s.beta, out, out2, out3, d, partial,
                                                       pstride, s.err);
  };
  // level 0 with two realizations per lane (k_lvl_op2) where the batch allows it
  auto lvl0 = [&](auto mode, const CUtensorMap& ta, const CUtensorMap& tb, const CUtensorMap& ta2,
                  const CUtensorMap& tb2, const float* b, const float* dinv, float* out, float* out2, float* out3,
                  float* d, double* partial, int pstride) {
    constexpr int kMode = decltype(mode)::value;
    if (B->pack) {
      auto k = mass ? k_lvl_op2<kMode, true> : k_lvl_op2<kMode, false>;
      // post-sweep: b (= r') and dinv of the own nodes come through the stage
      const CUtensorMap& tn2 = kMode == kLvlSmooth ? B->tm2_dinvo : B->tm2_dinv;
      const CUtensorMap& tbb = kMode == kLvlSmooth ? (even ? B->tm2_rBo : B->tm2_rAo) : tb2;
      k<<<B->grid2, kQThreads, LvlStage2<kMode>::kSmem, st>>>(
          B->L, B->MC2, ta2, tbb, tn2, B->tm2_e, B->tm2_d, B->tiles_j2, B->n_tiles2, B->n_items2, B->mask, b, dinv,
          om, s.alpha, s.beta, out, out2, out3, d, partial, pstride, s.err);
    } else {
      lvl(mode, B->L, B->MC, ta, tb, B->tm_dinvm, B->tm_em, B->tm_dm, B->tiles_jm, B->n_tiles_m, B->n_items_m,
          B->grid_m, B->mask, b, dinv, out, out2, out3, d, partial, pstride);
    }
  };
  // coarse level l: residual (out = b - A x) or post-sweep (out = x + omega dinv (b - A x)) of x into t
  auto lvlc = [&](auto mode, GmgLevel& g) {
    constexpr int kMode = decltype(mode)::value;
    if (B->pack) {
      auto k = mass ? k_lvl_op2<kMode, true> : k_lvl_op2<kMode, false>;
      k<<<g.grid2, kQThreads, LvlStage2<kMode>::kSmem, st>>>(
          g.L, g.MC2, g.tm2_x, g.tm2_bo, g.tm2_dinvo, g.tm2_e, g.tm2_x, g.tiles_j2, g.n_tiles2, g.n_items2, g.mask, g.b,
          g.dinv, om, s.alpha, s.beta, g.t, nullptr, nullptr, nullptr, nullptr, 1, s.err);
    } else {
      lvl(mode, g.L, g.MC, g.tm_x, g.tm_x, g.tm_x, g.tm_e, g.tm_x, g.tiles_j, g.n_tiles, g.n_items, g.grid, g.mask,
          g.b, kMode == kLvlSmooth ? g.dinv : nullptr, g.t, nullptr, nullptr, nullptr, nullptr, 1);
    }
  };
  using Start = std::integral_constant<int, kLvlStart>;
  using Resid = std::integral_constant<int, kLvlResid>;
  using Smooth = std::integral_constant<int, kLvlSmooth>;
  // level 0: r' = r - alpha q, qB = r' - A x0 with x0 = omega dinv r', partial r'.r'
  // (x0 itself is formed again by the level-0 prolongation)
  lvl0(Start{}, tm_rin, B->tm_qAm, even ? B->tm2_rA : B->tm2_rB, B->tm2_qA, nullptr, nullptr, qB, r_out, nullptr,
       nullptr, part2, 2);
  // down: restrict the residual, residual of the first sweep on every level but the coarsest
  for (int l = 1; l < nl; ++l) {
    GmgLevel& g = B->lv[l];
    const Lattice& Lf = l == 1 ? B->L : B->lv[l - 1].L;
    const float* tf = l == 1 ? qB : B->lv[l - 1].t;
    k_restrict<<<xfer_grid(g.L.n_int, Rp), xfer_block(Rp), 0, st>>>(Lf, g.L, g.interior, g.mask, tf, g.dinv, om, g.b,
                                                                     g.x);
    if (l < nl - 1) lvlc(Resid{}, g);
  }
  // coarsest level: the restriction made the first sweep; sweeps - 1 more, x and t alternating
  const float* res_c;
  if (B->lv[nl - 1].sweep_smem) {
    GmgLevel& g = B->lv[nl - 1];
    res_c = g.x;
    if (B->sweeps > 1) {
      auto k = mass ? k_coarse_sweeps<true> : k_coarse_sweeps<false>;
      k<<<Rp / 32, kMWarps * 32, g.sweep_smem, st>>>(g.L, g.MC, g.mask, g.b, g.dinv, g.E32, om, B->sweeps - 1, g.x,
                                                      g.t);
      res_c = g.t;
    }
  } else {
    GmgLevel& g = B->lv[nl - 1];
    bool in_x = true;
    for (int k = 1; k < B->sweeps; ++k) {
      lvl(Smooth{}, g.L, g.MC, in_x ? g.tm_x : g.tm_t, g.tm_x, g.tm_x, g.tm_e, g.tm_x, g.tiles_j, g.n_tiles,
          g.n_items, g.grid, g.mask, g.b, g.dinv, in_x ? g.t : g.x, nullptr, nullptr, nullptr, nullptr, 1);
      in_x = !in_x;
    }
    res_c = in_x ? g.x : g.t;
  }
  // up: prolongate into the level's iterate, one sweep (result in t)
  for (int l = nl - 2; l >= 1; --l) {
    GmgLevel& g = B->lv[l];
    k_prolong_add<<<prolong_grid(g.L.n_int, Rp), xfer_block(Rp), 0, st>>>(g.L, B->lv[l + 1].L, g.interior,
                                                                          g.L.n_int, g.mask, res_c, g.x, nullptr,
                                                                          nullptr, 0.f);
    lvlc(Smooth{}, g);
    res_c = g.t;
  }
  // level 0: x0 = omega dinv r' formed here (the start pass does not write it)
  k_prolong_add<<<prolong_grid(B->L.n_int, Rp), xfer_block(Rp), 0, st>>>(B->L, B->lv[1].L, B->interior,
                                                                          B->L.n_int, B->mask, res_c,
                                                                          B->xs.as<float>(), r_out,
                                                                          B->dinv.as<float>(), om);
  // level 0 post-sweep: z (into qB) and the partial z.r'
  lvl0(Smooth{}, B->tm_xs, B->tm_xs, B->tm2_xs, B->tm2_xs, r_out, B->dinv.as<float>(), qB, nullptr, nullptr, nullptr,
       part2 + 1, 2);
}

void gmg_iteration(BlockSys* B, const LoopCfg& c, int it, cudaStream_t st) {
  const int Rp = B->Rp;
  Scal& s = B->s;
  cudaEvent_t* ev = B->X.ev;
  const bool even = (it & 1) == 0;
  const int nt0 = B->pack ? B->n_tiles2 : B->n_tiles_m;
  double* part2 = B->part_op.as<double>();
  double* part1 = part2 + (size_t)2 * nt0 * Rp;
  float* p_out = even ? B->pB.as<float>() : B->p.as<float>();
  const CUtensorMap& tm_pin = even ? B->tm_pAm : B->tm_pBm;
  const bool mass = B->mass;
  if (it == 0) cudaEventRecordWithFlags(ev[6], st, cudaEventRecordExternal);
  gmg_vcycle(B, s, even, st);
  using PcgZ = std::integral_constant<int, kLvlPcgZ>;
  auto lvl0 = [&](auto mode, const CUtensorMap& ta, const CUtensorMap& tb, const CUtensorMap& ta2,
                  const CUtensorMap& tb2, float* out, float* out2, float* d, double* partial, int pstride) {
    constexpr int kMode = decltype(mode)::value;
    if (B->pack) {
      auto k = mass ? k_lvl_op2<kMode, true> : k_lvl_op2<kMode, false>;
      k<<<B->grid2, kQThreads, LvlStage2<kMode>::kSmem, st>>>(
          B->L, B->MC2, ta2, tb2, B->tm2_dinv, B->tm2_e, B->tm2_d, B->tiles_j2, B->n_tiles2, B->n_items2, B->mask,
          nullptr, nullptr, B->omega, s.alpha, s.beta, out, out2, nullptr, d, partial, pstride, s.err);
    } else {
      auto k = mass ? k_lvl_op<kMode, true> : k_lvl_op<kMode, false>;
      k<<<B->grid_m, kMThreads, LvlStage<kMode>::kSmem, st>>>(
          B->L, B->MC, ta, tb, B->tm_dinvm, B->tm_em, B->tm_dm, B->tiles_jm, B->n_tiles_m, B->n_items_m, B->mask,
          nullptr, nullptr, B->omega, s.alpha, s.beta, out, out2, nullptr, d, partial, pstride, s.err);
    }
  };
  cudaMemsetAsync(s.n_active, 0, 32, st);  // n_active and n_update
  k_gmg_beta<<<c.sblocks, 1024, 0, st>>>(Rp, nt0, part2, s, c.delta2, c.tol2);
  // p = z + beta p_old, d += alpha p_old, q = A p, partial p.q
  if (it == 0) cudaEventRecordWithFlags(ev[4], st, cudaEventRecordExternal);
  if (B->tc) {
    k_lvl_tc<kLvlPcgZ><<<B->grid_m, kMThreads, kTcSmem, st>>>(
        B->L, B->tc_bops.as<float>(), B->tm_qBm, tm_pin, B->tm_em, B->tm_dm, B->tiles_jm, B->n_tiles_m, B->n_items_m,
        B->mask, s.alpha, s.beta, B->q.as<float>(), p_out, B->d.as<float>(), part1, 1, s.err);
  } else {
    lvl0(PcgZ{}, B->tm_qBm, tm_pin, B->tm2_qB, even ? B->tm2_pA : B->tm2_pB, B->q.as<float>(), p_out,
         B->d.as<float>(), part1, 1);
  }
  if (it == 0) cudaEventRecordWithFlags(ev[5], st, cudaEventRecordExternal);
  k_gmg_alpha<<<c.sblocks, 1024, 0, st>>>(Rp, nt0, part1, s);
  if (it == 0) cudaEventRecordWithFlags(ev[7], st, cudaEventRecordExternal);
}

// Kernels of one multigrid iteration (for the launch count).
int gmg_launches(const BlockSys* B) {
  const int nl = B->n_lvl;
  const int coarse = B->lv[nl - 1].sweep_smem ? (B->sweeps > 1 ? 1 : 0) : B->sweeps - 1;
  return 1 + (nl - 1) + (nl - 2) + coarse + (nl - 1) + (nl - 2) + 1 + 1 + 1 + 1;
}

// The inner-loop graph of `chunk` FP32 iterations, kept in the exec slot and
// captured again only when one of its kernel arguments changes (FNV-1a over
// the argument bytes).
int block_graph(Context* ctx, BlockSys* B, const LoopCfg& c, cudaGraphExec_t* out) {
  const Lattice& L = B->L;
  const int Rp = B->Rp;
  cudaStream_t st = B->X.st;
  Scal& s = B->s;
  cudaEvent_t* ev = B->X.ev;
  const int* interior = B->interior;
  const uint8_t* mask = B->mask;
  WSlot &r32 = B->r32, &p = B->p, &q = B->q, &d = B->d, &dinv = B->dinv, &part_op = B->part_op,
        &part_up = B->part_up, &pB = B->pB, &rB = B->rB, &qB = B->qB;
  size_t key = 1469598103934665603ull;
  auto mix = [&key](const void* data, size_t n) {
    const unsigned char* bb = static_cast<const unsigned char*>(data);
    for (size_t i = 0; i < n; ++i) key = (key ^ bb[i]) * 1099511628211ull;
  };
  {
    const void* ptrs[] = {interior, mask, r32.ptr, p.ptr, q.ptr, d.ptr, dinv.ptr, part_op.ptr, part_up.ptr,
                          B->scal.ptr, pB.ptr, rB.ptr, qB.ptr, st};
    mix(ptrs, sizeof(ptrs));
    mix(&L, sizeof(L));
    mix(&B->MC, sizeof(B->MC));
    {
      const CUtensorMap* tms[9] = {&B->tm_rAm, &B->tm_rBm, &B->tm_qAm,   &B->tm_qBm, &B->tm_pAm,
                                   &B->tm_pBm, &B->tm_dinvm, &B->tm_em, &B->tm_dm};
      for (const CUtensorMap* t : tms) mix(t, sizeof(CUtensorMap));
    }
    const int mm[5] = {B->mass ? 1 : 0, B->n_tiles_m, B->n_items_m, B->grid_m, B->tiles_jm};
    mix(mm, sizeof(mm));
    const int gg[5] = {B->gmg ? 1 : 0, B->n_lvl, B->sweeps, B->pack ? 1 : 0, B->tc ? 1 : 0};
    mix(gg, sizeof(gg));
    if (B->gmg) {
      mix(&B->omega, sizeof(B->omega));
      mix(&B->xs.ptr, sizeof(void*));
      mix(&B->tm_xs, sizeof(CUtensorMap));
      for (int l = 1; l < B->n_lvl; ++l) mix(&B->lv[l], sizeof(GmgLevel));
      if (B->pack) {
        const CUtensorMap* t2[13] = {&B->tm2_rA, &B->tm2_rB, &B->tm2_qA, &B->tm2_qB, &B->tm2_pA,
                                     &B->tm2_pB, &B->tm2_xs, &B->tm2_dinv, &B->tm2_e, &B->tm2_d,
                                     &B->tm2_rAo, &B->tm2_rBo, &B->tm2_dinvo};
        for (const CUtensorMap* t : t2) mix(t, sizeof(CUtensorMap));
        mix(&B->MC2, sizeof(B->MC2));
      }
    }
    const double dd[2] = {c.delta2, c.tol2};
    mix(dd, sizeof(dd));
    const int ii[5] = {c.chunk, c.n_dir, B->n_upd, B->n_tiles, c.sblocks};
    mix(ii, sizeof(ii));
  }
  cudaGraphExec_t& gx = *B->X.graph;
  if (gx && *B->X.graph_key != key) {
    cudaGraphExecDestroy(gx);
    gx = nullptr;
  }
  if (!gx) {
    cudaGraph_t g;
    MSG_CUDA(ctx, cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    for (int it = 0; it < c.chunk; ++it) {
      // cudaEventRecordExternal: a real event-record node in the graph (plain
      // records during capture only order streams)
      if (B->gmg) {
        gmg_iteration(B, c, it, st);
      } else {
        // single-reduction loop: one operator launch per iteration; r, q and p
        // alternate between their two buffers
        const bool even = (it & 1) == 0;
        if (it == 0) cudaEventRecordWithFlags(ev[4], st, cudaEventRecordExternal);
        auto op = B->mass ? k_op_modal<true> : k_op_modal<false>;
        op<<<B->grid_m, kMThreads, kMSmem, st>>>(
            L, B->MC, even ? B->tm_rAm : B->tm_rBm, even ? B->tm_qAm : B->tm_qBm, even ? B->tm_pAm : B->tm_pBm,
            B->tm_dinvm, B->tm_em, B->tm_dm, B->tiles_jm, B->n_tiles_m, B->n_items_m, mask, s.alpha, s.beta,
            even ? rB.as<float>() : r32.as<float>(), even ? pB.as<float>() : p.as<float>(),
            even ? qB.as<float>() : q.as<float>(), d.as<float>(), part_op.as<double>(), s.err);
        if (it == 0) cudaEventRecordWithFlags(ev[5], st, cudaEventRecordExternal);
        cudaMemsetAsync(s.n_active, 0, 32, st);  // n_active and n_update
        if (it == 0) cudaEventRecordWithFlags(ev[6], st, cudaEventRecordExternal);
        k_alpha_gamma<<<c.sblocks, 1024, 0, st>>>(Rp, B->n_tiles_m, part_op.as<double>(), s, c.delta2, c.tol2);
        if (it == 0) cudaEventRecordWithFlags(ev[7], st, cudaEventRecordExternal);
      }
    }
    cudaError_t e = cudaStreamEndCapture(st, &g);
    if (e != cudaSuccess) return cuda_error(ctx, e, "capture inner chunk");
    e = cudaGraphInstantiate(&gx, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
      gx = nullptr;
      return cuda_error(ctx, e, "instantiate inner chunk");
    }
    *B->X.graph_key = key;
  }
  *out = gx;
  return MSG_OK;
}

// True-residual step (enqueued, not synchronised): x += d + alpha p, d = 0
// (unless first), r = b - A x in FP64, convergence and search-direction scalars.
int block_update(Context* ctx, BlockSys* B, const LoopCfg& c, const double* b, bool b_per_r, double tol, bool first,
                 int max_it, bool zero_x = false) {
  const Lattice& L = B->L;
  const int Rp = B->Rp;
  cudaStream_t st = B->X.st;
  Scal& s = B->s;
  const uint8_t* mask = B->mask;
  const float* dinv = B->dinv.as<float>();
  float* r32 = B->r32.as<float>();
  double* part = B->part_op.as<double>();
  if (zero_x) {
    // x = 0: r = b, and the partials ||b||^2, (dinv b).b of block_bnorm are the residual's
    k_b_to_r32<<<c.n_dir, 256, 0, st>>>(L.n_int, Rp, B->interior, b, b_per_r ? 1 : 0, r32);
    MSG_CUDA(ctx, cudaMemsetAsync(s.n_active, 0, 32, st));
    k_resid_scalars<<<c.sblocks, 1024, 0, st>>>(Rp, B->n_bsq, B->part_up.as<double>(), s, tol, first ? 1 : 0,
                                                 B->gmg ? 2 : 1, max_it);
    count_launch(ctx, 2);
    MSG_CUDA(ctx, cudaGetLastError());
    return MSG_OK;
  }
  {
    // x += d + alpha p (into the other x buffer) and the FP64 residual in one pass
    auto pick = [&](auto M, auto P, auto U) {
      return k_resid_modal<decltype(M)::value, decltype(P)::value, decltype(U)::value>;
    };
    using T1 = std::true_type;
    using F0 = std::false_type;
    const bool upd = !first;
    auto k = B->mass ? (b_per_r ? (upd ? pick(T1{}, T1{}, T1{}) : pick(T1{}, T1{}, F0{}))
                                : (upd ? pick(T1{}, F0{}, T1{}) : pick(T1{}, F0{}, F0{})))
                     : (b_per_r ? (upd ? pick(F0{}, T1{}, T1{}) : pick(F0{}, T1{}, F0{}))
                                : (upd ? pick(F0{}, F0{}, T1{}) : pick(F0{}, F0{}, F0{})));
    k<<<B->grid_r, kRThreads, kRSmem, st>>>(L, B->MCD, B->tm_xr, B->tm_dr, B->tm_pr, B->tm_er, B->tiles_jr,
                                             B->n_tiles_r, B->n_items_r, mask, b, dinv, s.alpha, B->xB.as<double>(),
                                             r32, part, s.err);
    if (upd) {
      MSG_CUDA(ctx, cudaMemsetAsync(B->d.ptr, 0, sizeof(float) * B->nvec, st));
      std::swap(B->x.ptr, B->xB.ptr);
      std::swap(B->tm_xr, B->tm_xBr);
    }
  }
  MSG_CUDA(ctx, cudaMemsetAsync(s.n_active, 0, 32, st));
  k_resid_scalars<<<c.sblocks, 1024, 0, st>>>(Rp, B->n_tiles_r, part, s, tol, first ? 1 : 0, B->gmg ? 2 : 1,
                                               max_it);
  count_launch(ctx, 2);
  MSG_CUDA(ctx, cudaGetLastError());
  return MSG_OK;
}

// ||b|| and (dinv b).b of every realization (b shared or per realization)
int block_bnorm(Context* ctx, BlockSys* B, const double* b, bool b_per_r) {
  cudaStream_t st = B->X.st;
  k_bsq<<<dim3(B->n_bsq, B->Rp / 32), 256, 0, st>>>(B->L.n_int, B->Rp, B->interior, b, b_per_r ? 1 : 0,
                                                   B->dinv.as<float>(), B->part_up.as<double>());
  k_bnorm<<<B->Rp / 32, 1024, 0, st>>>(B->R, B->Rp, B->n_bsq, B->part_up.as<double>(), B->s);
  count_launch(ctx, 2);
  return MSG_OK;
}

// The start of a batched solve (enqueued on the batch's stream): scalars,
// directions, the operator outputs and the correction zero (x too unless
// warm), ||b|| per realization, the loop's configuration and graph.
int block_solve_start(Context* ctx, BlockSys* B, const double* b, bool b_per_r, bool warm, double tol, int chunk_cap,
                      LoopCfg* c, cudaGraphExec_t* gexec) {
  cudaStream_t st = B->X.st;
  const size_t nvec = B->nvec;
  MSG_CUDA(ctx, cudaMemsetAsync(B->scal.ptr, 0, B->scal_bytes, st));
  if (!warm) MSG_CUDA(ctx, cudaMemsetAsync(B->x.ptr, 0, sizeof(double) * nvec, st));
  // directions, operator outputs and the correction start from zero
  const WSlot* z32[] = {&B->p, &B->q, &B->d, &B->pB, &B->qB};
  for (const WSlot* w : z32)
    if (w->ptr) MSG_CUDA(ctx, cudaMemsetAsync(w->ptr, 0, sizeof(float) * nvec, st));
  MSG_TRY(block_bnorm(ctx, B, b, b_per_r));
  *c = loop_cfg(ctx, B, tol, chunk_cap);
  MSG_TRY(block_graph(ctx, B, *c, gexec));
  return MSG_OK;
}

// Solve A x = b for every realization of the batch to the FP64 true relative
// residual tol: b is one vector (blat layout) or one per realization; x (slot 0)
// starts from zero, or from its content when warm. Per-realization results stay
// in B->s (its, res, done, breakdown); returns the batch status.
int block_solve(Context* ctx, BlockSys* B, const double* b, bool b_per_r, bool warm, int max_it, double tol,
                bool record_phases, int chunk_cap = 0) {
  NvtxRange range("msg: batched solve");
  cudaStream_t st = B->X.st;
  Scal& s = B->s;
  LoopCfg c;
  cudaGraphExec_t gexec = nullptr;
  MSG_TRY(block_solve_start(ctx, B, b, b_per_r, warm, tol, chunk_cap, &c, &gexec));
  cudaEvent_t* ev = B->X.ev;
  float t_resid = 0.f, t_inner = 0.f;

  int* h_flags = B->X.h_flags;  // [0] active, [4] update requests, [8] wait timeout (pinned)
  int status = MSG_OK;
  int total_inner = 0;
  int n_updates = 0;
  bool need_update = true, first = true;
  for (int guard = 0; guard < 1000000; ++guard) {
    if (need_update) {
      NvtxRange upd("msg: FP64 true residual");
      cudaEventRecord(ev[0], st);
      MSG_TRY(block_update(ctx, B, c, b, b_per_r, tol, first, 0x7fffffff, B->gmg && first && !warm));
      cudaEventRecord(ev[1], st);
      MSG_TRY(publish_flags(ctx, s.n_active, 9, h_flags, B->X.d_hflags, st));
      MSG_CUDA(ctx, cudaStreamSynchronize(st));
      float ms = 0.f;
      cudaEventElapsedTime(&ms, ev[0], ev[1]);
      t_resid += ms;
      first = false;
      ++n_updates;
      if (h_flags[0] == 0) break;  // every realization converged (or broke down)
    }
    if (total_inner >= max_it) {
      status = MSG_ERR_NOT_CONVERGED;
      break;
    }
    NvtxRange chunk_range("msg: FP32 inner chunk");
    cudaEventRecord(ev[2], st);
    cudaError_t e = cudaGraphLaunch(gexec, st);
    if (e != cudaSuccess) return cuda_error(ctx, e, "inner chunk");
    count_launch(ctx, (B->gmg ? gmg_launches(B) : 2) * c.chunk);
    total_inner += c.chunk;
    cudaEventRecord(ev[3], st);
    MSG_TRY(publish_flags(ctx, s.n_active, 9, h_flags, B->X.d_hflags, st));
    MSG_CUDA(ctx, cudaStreamSynchronize(st));
    float ms = 0.f, op_ms = 0.f, up_ms = 0.f;
    cudaEventElapsedTime(&ms, ev[2], ev[3]);
    t_inner += ms;
    if (B->X.ctx_stats && cudaEventElapsedTime(&op_ms, ev[4], ev[5]) == cudaSuccess &&
        cudaEventElapsedTime(&up_ms, ev[6], ev[7]) == cudaSuccess) {
      ctx->op_ms_sum += op_ms;
      ctx->upd_ms_sum += up_ms;
      ctx->op_samples += 1;
    }
    cudaGetLastError();
    // a realization that stopped iterating (breakdown) or asks for a check triggers an update
    if (h_flags[8]) {
      status = set_error(ctx, MSG_ERR_TIMEOUT, "a bounded wait of the staged operator expired");
      break;
    }
    need_update = B->fixed || (h_flags[4] > 0) || (h_flags[0] == 0);
  }
  if (B->X.ctx_stats) {
    if (record_phases) {
      ctx->t_phase[1] = t_inner;
      ctx->t_phase[3] = t_resid;
      ctx->t_phase[2] = (double)n_updates;
    } else {
      ctx->t_phase[1] += t_inner;
      ctx->t_phase[3] += t_resid;
      ctx->t_phase[2] += (double)n_updates;
    }
  }
  return status;
}

// Per-realization results of the last solve on the host; batch status.
int block_results(Context* ctx, BlockSys* B, int status, int* its_out, double* res_out) {
  const int Rp = B->Rp;
  cudaStream_t st = B->X.st;
  std::vector<int> its(Rp), brk(Rp), done(Rp);
  std::vector<double> res(Rp);
  MSG_CUDA(ctx, cudaMemcpyAsync(its.data(), B->s.its, sizeof(int) * Rp, cudaMemcpyDeviceToHost, st));
  MSG_CUDA(ctx, cudaMemcpyAsync(brk.data(), B->s.breakdown, sizeof(int) * Rp, cudaMemcpyDeviceToHost, st));
  MSG_CUDA(ctx, cudaMemcpyAsync(done.data(), B->s.done, sizeof(int) * Rp, cudaMemcpyDeviceToHost, st));
  MSG_CUDA(ctx, cudaMemcpyAsync(res.data(), B->s.res, sizeof(double) * Rp, cudaMemcpyDeviceToHost, st));
  MSG_CUDA(ctx, cudaStreamSynchronize(st));
  MSG_CUDA(ctx, cudaGetLastError());
  for (int r = 0; r < B->R; ++r) {
    if (its_out) its_out[r] = its[r];
    if (res_out) res_out[r] = res[r];
    if (!done[r] && status == MSG_OK) status = brk[r] == 1 ? MSG_ERR_BREAKDOWN : MSG_ERR_NOT_CONVERGED;
  }
  return status;
}

}  // namespace

int pc_matvec(Context* ctx, Mesh* m, double nu, const MSG_KL* kl, int mo, int po, const double* u_host,
              double* y_host) {
  if (!m->structured) return set_error(ctx, MSG_ERR_NOT_STRUCTURED, "the Galerkin product needs a structured lattice");
  if (!kl->gaussian) return set_error(ctx, MSG_ERR_INVALID_ARGUMENT, "the Galerkin product needs a Gaussian KL field");
  if (mo < 1 || po < 1 || mo > kl->n_terms)
    return set_error(ctx, MSG_ERR_INVALID_ARGUMENT, "polynomial chaos: need 1 <= m <= n_terms and p >= 1");
  std::vector<int> tptr, tpos, tk;
  std::vector<double> tc;
  MSG_TRY(pc_gaussian_terms(mo, po, tptr, tpos, tk, tc));
  const int P = (int)tptr.size() - 1;
  const int Pp = (P + 31) / 32 * 32, Mp = mo + 1;
  cudaStream_t st = ctx->stream;
  double K576[576];
  MSG_TRY(unit_cube_khat(ctx, m->h, nu, K576));
  KhatD KD;
  for (int c = 0; c < kKhatClasses; ++c) KD.v[c] = K576[kKhatRep[c]];
  KLDevice kd;
  MSG_TRY(kl_prepare(ctx, m, kl, &kd));
  const size_t npad = (size_t)m->NXp * m->NYp * m->NZp;
  DevMem dE, du, dy, dlat_u, dlat_y, dptr, dpos, dk, dc;
  MSG_TRY(dE.alloc(ctx, sizeof(double) * npad * Mp));
  MSG_TRY(du.alloc(ctx, sizeof(double) * (size_t)P * std::max(1, m->n_dofs)));
  MSG_TRY(dy.alloc(ctx, sizeof(double) * (size_t)P * std::max(1, m->n_dofs)));
  MSG_TRY(dlat_u.alloc(ctx, sizeof(double) * npad * 3 * Pp));
  MSG_TRY(dlat_y.alloc(ctx, sizeof(double) * npad * 3 * Pp));
  MSG_TRY(dptr.alloc(ctx, sizeof(int) * tptr.size()));
  MSG_TRY(dpos.alloc(ctx, sizeof(int) * std::max<size_t>(1, tpos.size())));
  MSG_TRY(dk.alloc(ctx, sizeof(int) * std::max<size_t>(1, tk.size())));
  MSG_TRY(dc.alloc(ctx, sizeof(double) * std::max<size_t>(1, tc.size())));
  MSG_CUDA(ctx, cudaMemcpyAsync(dptr.ptr, tptr.data(), sizeof(int) * tptr.size(), cudaMemcpyHostToDevice, st));
  MSG_CUDA(ctx, cudaMemcpyAsync(dpos.ptr, tpos.data(), sizeof(int) * tpos.size(), cudaMemcpyHostToDevice, st));
  MSG_CUDA(ctx, cudaMemcpyAsync(dk.ptr, tk.data(), sizeof(int) * tk.size(), cudaMemcpyHostToDevice, st));
  MSG_CUDA(ctx, cudaMemcpyAsync(dc.ptr, tc.data(), sizeof(double) * tc.size(), cudaMemcpyHostToDevice, st));
  MSG_CUDA(ctx, cudaMemcpyAsync(du.ptr, u_host, sizeof(double) * (size_t)P * m->n_dofs, cudaMemcpyHostToDevice, st));
  MSG_CUDA(ctx, cudaMemsetAsync(dE.ptr, 0, sizeof(double) * npad * Mp, st));
  MSG_CUDA(ctx, cudaMemsetAsync(dlat_u.ptr, 0, sizeof(double) * npad * 3 * Pp, st));
  MSG_CUDA(ctx, cudaMemsetAsync(dlat_y.ptr, 0, sizeof(double) * npad * 3 * Pp, st));
  k_pc_fields<<<(m->n_elems + 127) / 128, 128, 0, st>>>(m->n_elems, mo, Mp, kl->mean, kd.psi,
                                                        m->d_pad_elem_row.as<int>(), dE.as<double>());
  const dim3 gd((m->n_dofs + 255) / 256, P);
  if (m->n_dofs > 0)
    k_pc_scatter<<<gd, 256, 0, st>>>(m->n_dofs, P, Pp, m->d_pad_free_rows.as<int>(), du.as<double>(),
                                     dlat_u.as<double>());
  Lattice L;
  L.NX = m->nx + 1; L.NY = m->ny + 1; L.NZ = m->nz + 1;
  L.NXp = m->NXp; L.NYp = m->NYp; L.NZp = m->NZp;
  L.Rp = Pp;
  L.tiles_j = (L.NY + kTJ - 1) / kTJ;
  L.n_pad = (int)npad;
  L.n_int = L.NX * L.NY * L.NZ;
  const int n_tiles = L.tiles_j * ((L.NZ + kTK - 1) / kTK);
  k_pc_matvec<<<dim3(n_tiles, Pp / 32), dim3(32, kWarps), 0, st>>>(
      L, KD, dlat_u.as<double>(), dE.as<double>(), Mp, m->d_pad_mask.as<uint8_t>(), dptr.as<int>(), dpos.as<int>(),
      dk.as<int>(), dc.as<double>(), P, dlat_y.as<double>());
  if (m->n_dofs > 0)
    k_pc_gather<<<gd, 256, 0, st>>>(m->n_dofs, P, Pp, m->d_pad_free_rows.as<int>(), dlat_y.as<double>(),
                                    dy.as<double>());
  count_launch(ctx, 4);
  MSG_CUDA(ctx, cudaGetLastError());
  MSG_CUDA(ctx, cudaMemcpyAsync(y_host, dy.ptr, sizeof(double) * (size_t)P * m->n_dofs, cudaMemcpyDeviceToHost, st));
  MSG_CUDA(ctx, cudaStreamSynchronize(st));
  return MSG_OK;
}

int wait_selftest(Context* ctx, long polls, int* expired) {
  DevMem flag;
  MSG_TRY(flag.alloc(ctx, sizeof(int)));
  MSG_CUDA(ctx, cudaMemsetAsync(flag.ptr, 0, sizeof(int), ctx->stream));
  k_wait_selftest<<<1, 32, 0, ctx->stream>>>(polls, flag.as<int>());
  count_launch(ctx, 1);
  int h = 0;
  MSG_CUDA(ctx, cudaMemcpyAsync(&h, flag.ptr, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  MSG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  MSG_CUDA(ctx, cudaGetLastError());
  *expired = h;
  return MSG_OK;
}

int block_mixed_solve(Context* ctx, Mesh* m, double nu, const KLDevice* kl, const double* d_xi, int R, int Rp,
                      const double* d_b_dof, int max_it, double tol, int tip_dof, double* d_X, BatchOut out) {
  BlockSys B;
  MSG_TRY(block_setup(ctx, m, nu, 1.0, 1.0, 0.0, R, Rp, &B));
  B.fixed = ctx->fixed_updates != 0;
  cudaStream_t st = ctx->stream;
  MSG_TRY(block_field(ctx, m, &B, kl, d_xi));
  // b in lattice layout (one load vector for the whole batch)
  k_lattice_rhs<<<(m->n_dofs + 255) / 256, 256, 0, st>>>(m->n_dofs, m->d_pad_free_rows.as<int>(), d_b_dof,
                                                         B.blat.as<double>());
  count_launch(ctx);
  MSG_CUDA(ctx, cudaStreamSynchronize(st));
  float fms = 0.f;
  cudaEventElapsedTime(&fms, ctx->ev[10], ctx->ev[11]);
  ctx->t_phase[0] = fms;
  int status = block_solve(ctx, &B, B.blat.as<double>(), false, false, max_it, tol, true);
  if (status == MSG_ERR_TIMEOUT) return status;

  // outputs
  if (d_X) {
    dim3 g((m->n_dofs + 31) / 32, Rp / 32);
    k_gather_solution<<<g, dim3(32, 8), 0, st>>>(m->n_dofs, R, Rp, m->d_pad_free_rows.as<int>(), B.x.as<double>(),
                                                 d_X);
    count_launch(ctx);
  }
  WSlot tipbuf;
  if (out.tip && tip_dof >= 0 && tip_dof < m->n_dofs) {
    int row = 0;
    MSG_CUDA(ctx, cudaMemcpyAsync(&row, m->d_pad_free_rows.as<int>() + tip_dof, sizeof(int), cudaMemcpyDeviceToHost,
                                  st));
    MSG_CUDA(ctx, cudaStreamSynchronize(st));
    MSG_TRY(workspace(ctx, 17, sizeof(double) * Rp, &tipbuf.ptr));
    k_gather_tip<<<(R + 127) / 128, 128, 0, st>>>(R, Rp, row, B.x.as<double>(), tipbuf.as<double>());
    count_launch(ctx);
    MSG_CUDA(ctx, cudaMemcpyAsync(out.tip, tipbuf.ptr, sizeof(double) * R, cudaMemcpyDeviceToHost, st));
  }
  status = block_results(ctx, &B, status, out.iterations, out.rel_res);
  if (status != MSG_OK)
    return set_error(ctx, status, "mixed batched solve: %s",
                     status == MSG_ERR_BREAKDOWN ? "PCG breakdown" : "not converged");
  return MSG_OK;
}

LatticeRunner::~LatticeRunner() {
  if (st) cudaStreamSynchronize(st);
  if (graph) cudaGraphExecDestroy(graph);
  for (cudaEvent_t& e : ev)
    if (e) cudaEventDestroy(e);
  if (st) cudaStreamDestroy(st);
  delete[] pool;
}

// Several cube-lattice batches side by side. Each batch has its own stream,
// events, flag words (mapped words 512 + 16 k of the context's), loop graph and
// buffer set (ctx->lat_runners[k]); the set-ups run on the context's stream one
// after another (the KL table's device copy is the context's). Then one host
// thread steps every batch's loop in turn: a round enqueues the next step of
// every running batch (its FP64 true residual or a chunk of iterations, then
// its flags) before it waits for any, so that one batch's host round trip and
// small launches overlap the other batches' kernels. Each batch takes exactly
// the steps block_solve takes for it alone, so its results are the same.
int block_mixed_solve_many(Context* ctx, std::vector<LatticeJob>& jobs, int max_it, double tol,
                           const std::function<int()>& alongside) {
  NvtxRange range("msg: cube-lattice batches side by side");
  const int n = (int)jobs.size();
  constexpr int kMaxSideBySide = 32;  // flag words 512 ... 1023 of the context's 1024
  if (n > kMaxSideBySide)
    return set_error(ctx, MSG_ERR_INVALID_ARGUMENT, "at most %d cube lattices side by side", kMaxSideBySide);
  MSG_TRY(context_resources(ctx));
  while ((int)ctx->lat_runners.size() < n) {
    std::unique_ptr<LatticeRunner> r(new LatticeRunner());
    MSG_CUDA(ctx, cudaStreamCreateWithFlags(&r->st, cudaStreamNonBlocking));
    for (cudaEvent_t& e : r->ev) MSG_CUDA(ctx, cudaEventCreate(&e));
    r->pool = new DevMem[kWorkSlots];
    ctx->lat_runners.push_back(r.release());
  }
  std::vector<std::unique_ptr<BlockSys>> Bs(n);
  std::vector<LoopCfg> cfg(n);
  std::vector<cudaGraphExec_t> gx(n, nullptr);
  cudaStream_t cs = ctx->stream;
  for (int i = 0; i < n; ++i) {
    LatticeJob& J = jobs[i];
    LatticeRunner* run = ctx->lat_runners[i];
    if (!J.m->structured) return set_error(ctx, MSG_ERR_NOT_STRUCTURED, "mesh is not a structured cube lattice");
    BlockExec X;
    X.st = run->st;
    X.ev = run->ev;
    X.h_flags = ctx->h_flags + 512 + 16 * i;
    X.d_hflags = ctx->d_hflags ? ctx->d_hflags + 512 + 16 * i : nullptr;
    X.graph = &run->graph;
    X.graph_key = &run->graph_key;
    X.ctx_stats = false;
    Bs[i].reset(new BlockSys());
    BlockSys* B = Bs[i].get();
    const int Rp = (J.R + 63) / 64 * 64;
    MSG_TRY(block_setup(ctx, J.m, J.nu, 1.0, 1.0, 0.0, J.R, Rp, B, run->pool, &X));
    B->fixed = ctx->fixed_updates != 0;
    MSG_CUDA(ctx, cudaStreamSynchronize(run->st));
    KLDevice kd;
    MSG_TRY(kl_prepare(ctx, J.m, J.kl, &kd));
    MSG_TRY(block_field(ctx, J.m, B, &kd, J.d_xi));
    k_lattice_rhs<<<(J.m->n_dofs + 255) / 256, 256, 0, cs>>>(J.m->n_dofs, J.m->d_pad_free_rows.as<int>(), J.d_b,
                                                             B->blat.as<double>());
    count_launch(ctx);
    MSG_CUDA(ctx, cudaStreamSynchronize(cs));  // before the next batch's KL table replaces this one's
    MSG_TRY(block_solve_start(ctx, B, B->blat.as<double>(), false, false, tol, 0, &cfg[i], &gx[i]));
    if (J.h_tip && run->tip.bytes < sizeof(double) * Rp) {
      run->tip.release();
      MSG_TRY(run->tip.alloc(ctx, sizeof(double) * Rp));
    }
  }
  // the loops, stepped in turn (block_solve's decisions, batch by batch), and
  // the outputs: on a second host thread while `alongside` runs on this one
  auto run_loops = [&]() -> int {
  struct Step {
    bool need_update = true, first = true, live = true;
    int total_inner = 0, status = MSG_OK, kind = 0;  // kind: 1 true residual, 2 chunk
  };
  std::vector<Step> sp(n);
  for (int round = 0; round < 1000000; ++round) {
    bool any = false;
    for (int i = 0; i < n; ++i) {
      Step& u = sp[i];
      if (!u.live) continue;
      BlockSys* B = Bs[i].get();
      if (u.need_update) {
        u.kind = 1;
        MSG_TRY(block_update(ctx, B, cfg[i], B->blat.as<double>(), false, tol, u.first, 0x7fffffff,
                             B->gmg && u.first));
      } else {
        u.kind = 2;
        const cudaError_t e = cudaGraphLaunch(gx[i], B->X.st);
        if (e != cudaSuccess) return cuda_error(ctx, e, "inner chunk");
        count_launch(ctx, (B->gmg ? gmg_launches(B) : 2) * cfg[i].chunk);
        u.total_inner += cfg[i].chunk;
      }
      MSG_TRY(publish_flags(ctx, B->s.n_active, 9, B->X.h_flags, B->X.d_hflags, B->X.st));
      any = true;
    }
    if (!any) break;
    for (int i = 0; i < n; ++i) {
      Step& u = sp[i];
      if (!u.live) continue;
      BlockSys* B = Bs[i].get();
      MSG_CUDA(ctx, cudaStreamSynchronize(B->X.st));
      const int* h = B->X.h_flags;
      if (u.kind == 1) {
        u.first = false;
        if (h[0] == 0) {  // every realization converged (or broke down)
          u.live = false;
          continue;
        }
        u.need_update = false;
      } else {
        if (h[8]) {
          u.status = set_error(ctx, MSG_ERR_TIMEOUT, "a bounded wait of the staged operator expired");
          u.live = false;
          continue;
        }
        u.need_update = B->fixed || (h[4] > 0) || (h[0] == 0);
      }
      if (!u.need_update && u.total_inner >= max_it) {
        u.status = MSG_ERR_NOT_CONVERGED;
        u.live = false;
      }
    }
  }
  // outputs, batch by batch
  for (int i = 0; i < n; ++i) {
    LatticeJob& J = jobs[i];
    BlockSys* B = Bs[i].get();
    cudaStream_t st = B->X.st;
    Mesh* m = J.m;
    int status = sp[i].status;
    if (status == MSG_ERR_TIMEOUT) {
      J.status = status;
      continue;
    }
    if (J.d_X) {
      dim3 g((m->n_dofs + 31) / 32, B->Rp / 32);
      k_gather_solution<<<g, dim3(32, 8), 0, st>>>(m->n_dofs, J.R, B->Rp, m->d_pad_free_rows.as<int>(),
                                                   B->x.as<double>(), J.d_X);
      count_launch(ctx);
    }
    if (J.h_tip && J.tip_dof >= 0 && J.tip_dof < m->n_dofs) {
      int row = 0;
      MSG_CUDA(ctx, cudaMemcpyAsync(&row, m->d_pad_free_rows.as<int>() + J.tip_dof, sizeof(int),
                                    cudaMemcpyDeviceToHost, st));
      MSG_CUDA(ctx, cudaStreamSynchronize(st));
      DevMem& tip = ctx->lat_runners[i]->tip;  // sized in the set-up
      k_gather_tip<<<(J.R + 127) / 128, 128, 0, st>>>(J.R, B->Rp, row, B->x.as<double>(), tip.as<double>());
      count_launch(ctx);
      MSG_CUDA(ctx, cudaMemcpyAsync(J.h_tip, tip.ptr, sizeof(double) * J.R, cudaMemcpyDeviceToHost, st));
    }
    status = block_results(ctx, B, status, J.h_its, J.h_res);  // synchronises the batch's stream
    if (status != MSG_OK)
      set_error(ctx, status, "mixed batched solve: %s", status == MSG_ERR_BREAKDOWN ? "PCG breakdown" : "not converged");
    J.status = status;
  }
  for (int i = 0; i < n; ++i) MSG_CUDA(ctx, cudaStreamSynchronize(ctx->lat_runners[i]->st));
  return MSG_OK;
  };
  if (!alongside) return run_loops();
  int loop_status = MSG_OK;
  std::thread worker([&] {
    const cudaError_t e = cudaSetDevice(ctx->device);
    loop_status = e == cudaSuccess ? run_loops() : cuda_error(ctx, e, "cudaSetDevice");
  });
  struct Join {  // joined on every way out, an exception from `alongside` included
    std::thread& t;
    ~Join() {
      if (t.joinable()) t.join();
    }
  } join{worker};
  const int a_status = alongside();
  worker.join();
  return loop_status != MSG_OK ? loop_status : a_status;
}

int block_newmark(Context* ctx, Mesh* m, double nu, const KLDevice* kl, const double* d_xi, int R, int Rp,
                  const NewmarkParams& nm, const double* d_f_dof, int max_it, double tol, int tip_dof,
                  double* tip_hist, double* d_U, int* its_total) {
  if (nm.delta < 0.5) return set_error(ctx, MSG_ERR_INVALID_ARGUMENT, "Newmark delta has to be bigger than 0.5");
  const double a_limit = 0.25 * (0.5 + nm.delta) * (0.5 + nm.delta);
  if (nm.alpha < a_limit)
    return set_error(ctx, MSG_ERR_INVALID_ARGUMENT, "Newmark alpha has to be bigger than %g", a_limit);
  if (!(nm.dt > 0) || nm.n_steps < 0 || nm.acc_dir < 0 || nm.acc_dir > 2)
    return set_error(ctx, MSG_ERR_INVALID_ARGUMENT, "invalid Newmark time step, step count or load direction");
  // NewmarkDynamicAnalyzer.InitializeCoefficients
  const double dt = nm.dt;
  const double a0 = 1 / (nm.alpha * dt * dt), a1 = nm.delta / (nm.alpha * dt), a2 = 1 / (nm.alpha * dt);
  const double a3 = 1 / (2 * nm.alpha) - 1, a4 = nm.delta / nm.alpha - 1, a5 = dt * 0.5 * (nm.delta / nm.alpha - 2);
  const double a6 = dt * (1 - nm.delta), a7 = nm.delta * dt;
  // effective matrix K + a0 M + a1 (alpha_R M + beta_R K)
  const double cK = 1.0 + a1 * nm.ray_beta, cM = a0 + a1 * nm.ray_alpha;
  BlockSys B;
  MSG_TRY(block_setup(ctx, m, nu, nm.rho, cK, cM, R, Rp, &B));
  MSG_TRY(block_field(ctx, m, &B, kl, d_xi));
  cudaStream_t st = ctx->stream;
  const Lattice& L = B.L;
  const size_t nvec = B.nvec, npad = B.npad;
  // state and right-hand-side buffers (batch layout, FP64): u, v, a, w1, w2, rhs; fM, f (shared)
  WSlot u, v, a, w1, w2, rhs, fM, fst, hist;
  MSG_TRY(workspace(ctx, 21, sizeof(double) * nvec, &u.ptr));
  MSG_TRY(workspace(ctx, 22, sizeof(double) * nvec, &v.ptr));
  MSG_TRY(workspace(ctx, 23, sizeof(double) * nvec, &a.ptr));
  MSG_TRY(workspace(ctx, 24, sizeof(double) * nvec, &w1.ptr));
  MSG_TRY(workspace(ctx, 25, sizeof(double) * nvec, &w2.ptr));
  MSG_TRY(workspace(ctx, 26, sizeof(double) * nvec, &rhs.ptr));
  MSG_TRY(workspace(ctx, 27, sizeof(double) * npad * 3, &fM.ptr));
  MSG_TRY(workspace(ctx, 28, sizeof(double) * npad * 3, &fst.ptr));
  MSG_TRY(workspace(ctx, 29, sizeof(double) * (size_t)std::max(1, nm.n_steps) * Rp, &hist.ptr));
  const WSlot* zs[] = {&u, &v, &a, &w1, &w2, &rhs};
  for (const WSlot* w : zs) MSG_CUDA(ctx, cudaMemsetAsync(w->ptr, 0, sizeof(double) * nvec, st));
  MSG_CUDA(ctx, cudaMemsetAsync(fst.ptr, 0, sizeof(double) * npad * 3, st));
  MSG_CUDA(ctx, cudaMemsetAsync(hist.ptr, 0, sizeof(double) * (size_t)std::max(1, nm.n_steps) * Rp, st));
  if (d_f_dof)
    k_lattice_rhs<<<(m->n_dofs + 255) / 256, 256, 0, st>>>(m->n_dofs, m->d_pad_free_rows.as<int>(), d_f_dof,
                                                           fst.as<double>());
  // inertial load pattern fM = Mhat-assembled unit acceleration in acc_dir at every node
  // (Hexa8.CalculateAccelerationForces), one column of M applied to the unit field
  KhatD kzero;
  for (int c = 0; c < kKhatClasses; ++c) kzero.v[c] = 0.0;
  MassClasses<double> m1;
  for (int i = 0; i < 4; ++i) m1.v[i] = B.cM != 0.0 ? B.MD.v[i] / B.cM : 0.0;
  const dim3 op_grid(B.n_tiles, Rp / 32), op_block(32, kWarps);
  const int ew = ctx->sm_count * 8;
  k_unit_dir<<<ew, 256, 0, st>>>(L.n_int, Rp, B.interior, nm.acc_dir, w1.as<double>());
  k_apply64<false><<<op_grid, op_block, 0, st>>>(L, kzero, m1, w1.as<double>(), B.E64.as<double>(), w2.as<double>());
  k_column<<<ew, 256, 0, st>>>(npad * 3, Rp, 0, w2.as<double>(), fM.as<double>());
  MSG_CUDA(ctx, cudaMemsetAsync(w1.ptr, 0, sizeof(double) * nvec, st));
  count_launch(ctx, d_f_dof ? 4 : 3);
  // RHS operators: M (w1) and beta_R E Khat (w2)
  KhatD kbeta;
  for (int c = 0; c < kKhatClasses; ++c) kbeta.v[c] = (B.cK != 0.0 ? B.KD.v[c] / B.cK : 0.0) * nm.ray_beta;
  MassClasses<double> mzero;
  for (int i = 0; i < 4; ++i) mzero.v[i] = 0.0;
  int row = -1;
  if (tip_dof >= 0 && tip_dof < m->n_dofs) {
    MSG_CUDA(ctx, cudaMemcpyAsync(&row, m->d_pad_free_rows.as<int>() + tip_dof, sizeof(int), cudaMemcpyDeviceToHost,
                                  st));
    MSG_CUDA(ctx, cudaStreamSynchronize(st));
  }
  const double two_pi = 2.0 * 3.14159265358979323846;
  int status = MSG_OK;
  std::vector<int> its(Rp);
  if (its_total) std::fill(its_total, its_total + R, 0);
  ctx->t_phase[1] = ctx->t_phase[2] = ctx->t_phase[3] = 0.0;
  for (int i = 0; i < nm.n_steps; ++i) {
    const double ag = nm.acc_amp * std::sin(two_pi / nm.acc_period * dt * i);
    // uu = a0 u + a2 v + a3 a, uc = a1 u + a4 v + a5 a; M uu + C uc = M (uu + alpha_R uc) + beta_R K uc
    k_nm_pre<<<ew, 256, 0, st>>>(L.n_int, Rp, B.interior, u.as<double>(), v.as<double>(), a.as<double>(),
                                 a0 + nm.ray_alpha * a1, a2 + nm.ray_alpha * a4, a3 + nm.ray_alpha * a5, a1, a4, a5,
                                 w1.as<double>(), w2.as<double>());
    k_apply64<false><<<op_grid, op_block, 0, st>>>(L, kzero, m1, w1.as<double>(), B.E64.as<double>(),
                                                   rhs.as<double>());
    k_apply64<true><<<op_grid, op_block, 0, st>>>(L, kbeta, mzero, w2.as<double>(), B.E64.as<double>(),
                                                  rhs.as<double>());
    k_nm_rhs<<<ew, 256, 0, st>>>(L.n_int, Rp, B.interior, B.mask, d_f_dof ? fst.as<double>() : nullptr,
                                 fM.as<double>(), ag, rhs.as<double>());
    // start from the Newmark predictor of the new displacement (newmark_predictor = 1),
    // or from the last displacement
    if (ctx->nm_predictor) {
      k_nm_predict<<<ew, 256, 0, st>>>(nvec, u.as<double>(), v.as<double>(), a.as<double>(), dt,
                                       (0.5 - nm.alpha) * dt * dt, B.x.as<double>());
      count_launch(ctx);
    } else {
      MSG_CUDA(ctx, cudaMemcpyAsync(B.x.ptr, u.ptr, sizeof(double) * nvec, cudaMemcpyDeviceToDevice, st));
    }
    count_launch(ctx, 4);
    // a few iterations per step: short graph chunks keep the host checks close
    status = block_solve(ctx, &B, rhs.as<double>(), true, true, max_it, tol, false, 4);
    if (status == MSG_ERR_TIMEOUT) return status;
    status = block_results(ctx, &B, status, its.data(), nullptr);
    if (status != MSG_OK)
      return set_error(ctx, status, "Newmark step %d: %s", i,
                       status == MSG_ERR_BREAKDOWN ? "PCG breakdown" : "not converged");
    if (its_total)
      for (int r = 0; r < R; ++r) its_total[r] += its[r];
    k_nm_post<<<ew, 256, 0, st>>>(L.n_int, Rp, B.interior, B.x.as<double>(), u.as<double>(), v.as<double>(),
                                  a.as<double>(), a0, a2, a3, a6, a7);
    count_launch(ctx);
    if (row >= 0) {
      k_gather_tip<<<(R + 127) / 128, 128, 0, st>>>(R, Rp, row, u.as<double>(), hist.as<double>() + (size_t)i * Rp);
      count_launch(ctx);
    }
  }
  if (d_U) {
    dim3 g((m->n_dofs + 31) / 32, Rp / 32);
    k_gather_solution<<<g, dim3(32, 8), 0, st>>>(m->n_dofs, R, Rp, m->d_pad_free_rows.as<int>(), u.as<double>(),
                                                 d_U);
    count_launch(ctx);
  }
  if (tip_hist && nm.n_steps > 0) {
    std::vector<double> h((size_t)nm.n_steps * Rp);
    MSG_CUDA(ctx, cudaMemcpyAsync(h.data(), hist.ptr, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, st));
    MSG_CUDA(ctx, cudaStreamSynchronize(st));
    for (int r = 0; r < R; ++r)
      for (int i = 0; i < nm.n_steps; ++i) tip_hist[(size_t)r * nm.n_steps + i] = h[(size_t)i * Rp + r];
  }
  MSG_CUDA(ctx, cudaStreamSynchronize(st));
  MSG_CUDA(ctx, cudaGetLastError());
  return MSG_OK;
}

// ---------------------------------------------------------------- serving lanes
// A lane is one model (mesh, material, KL table, load) with `capacity`
// realization slots that requests enter and leave at chunk boundaries
// (continuous batching). The FP64 true-residual step runs after every chunk
// for every slot, and a slot's first step treats it as a new system, so a
// request's arithmetic is the same whatever else shares the lane. It owns its
// memory, stream, events, pinned flags and inner-loop graph.
struct Lane {
  Context* ctx = nullptr;
  Mesh* m = nullptr;
  BlockSys B;
  DevMem own[kWorkSlots];
  DevMem psi, d_xi, d_slots, d_col;
  KLDevice kd;
  cudaStream_t st = nullptr;
  cudaEvent_t ev[12] = {nullptr};
  int* h_flags = nullptr;        // pinned 64 B
  int* h_state = nullptr;        // pinned: act, done, its, breakdown, fresh [Rp each]
  double* h_res = nullptr;       // pinned [Rp]
  double* h_xi = nullptr;        // pinned [capacity][n_terms]
  int* h_slots = nullptr;        // pinned [capacity]
  double* h_col = nullptr;       // pinned [n_dofs]
  cudaGraphExec_t graph = nullptr;
  size_t graph_key = 0;
  LoopCfg cfg;
  int capacity = 0, n_terms = 0, max_it = 0, n_pending = 0;
  double tol = 1e-8;
  ~Lane() {
    if (st) cudaStreamSynchronize(st);
    if (graph) cudaGraphExecDestroy(graph);
    for (auto& e : ev)
      if (e) cudaEventDestroy(e);
    void* pins[] = {h_flags, h_state, h_res, h_xi, h_slots, h_col};
    for (void* p : pins)
      if (p) cudaFreeHost(p);
    if (st) cudaStreamDestroy(st);
    if (m) release(m);
  }
};

int lane_create(Context* ctx, Mesh* m, double nu, const MSG_KL* kl, const double* b_host, int capacity, double tol,
                int max_it, Lane** out) {
  if (!m->structured) return set_error(ctx, MSG_ERR_NOT_STRUCTURED, "serving needs a structured cube lattice");
  if (capacity <= 0 || !(tol > 0) || max_it <= 0)
    return set_error(ctx, MSG_ERR_INVALID_ARGUMENT, "serving lane: invalid capacity, tolerance or iteration limit");
  std::unique_ptr<Lane> L(new Lane());
  L->ctx = ctx;
  L->m = m;
  retain(m);
  const int Rp = (capacity + 63) / 64 * 64;  // 64-wide groups: the packed level operator
  L->capacity = Rp;
  L->tol = tol;
  L->max_it = max_it;
  L->n_terms = kl->n_terms;
  MSG_CUDA(ctx, cudaSetDevice(ctx->device));
  // smaller models get higher stream priority: their short launches are
  // scheduled between the work items of larger models' launches
  int prio_least = 0, prio_greatest = 0;
  MSG_CUDA(ctx, cudaDeviceGetStreamPriorityRange(&prio_least, &prio_greatest));
  const double lg = std::log2((double)std::max(1, m->n_nodes));
  const double f = std::min(1.0, std::max(0.0, (lg - std::log2(729.0)) / (std::log2(117649.0) - std::log2(729.0))));
  const int prio = ctx->serve_priority ? prio_greatest + (int)std::lround(f * (prio_least - prio_greatest))
                                       : prio_least;
  MSG_CUDA(ctx, cudaStreamCreateWithPriority(&L->st, cudaStreamNonBlocking, prio));
  for (auto& e : L->ev) MSG_CUDA(ctx, cudaEventCreate(&e));
  MSG_CUDA(ctx, cudaMallocHost(&L->h_flags, 64));
  MSG_CUDA(ctx, cudaMallocHost(&L->h_state, sizeof(int) * 5 * Rp));
  MSG_CUDA(ctx, cudaMallocHost(&L->h_res, sizeof(double) * Rp));
  MSG_CUDA(ctx, cudaMallocHost(&L->h_xi, sizeof(double) * (size_t)Rp * kl->n_terms));
  MSG_CUDA(ctx, cudaMallocHost(&L->h_slots, sizeof(int) * Rp));
  MSG_CUDA(ctx, cudaMallocHost(&L->h_col, sizeof(double) * (size_t)std::max(1, m->n_dofs)));
  std::memset(L->h_flags, 0, 64);
  BlockExec X;
  X.st = L->st;
  X.ev = L->ev;
  X.h_flags = L->h_flags;
  X.graph = &L->graph;
  X.graph_key = &L->graph_key;
  X.ctx_stats = false;
  X.persistent = ctx->serve_persistent != 0;
  MSG_TRY(block_setup(ctx, m, nu, 1.0, 1.0, 0.0, Rp, Rp, &L->B, L->own, &X));
  L->B.fixed = true;
  // KL table -> psi (own copy: the context's KL workspace is reused by other calls)
  KLDevice kd;
  MSG_TRY(kl_prepare(ctx, m, kl, &kd));
  MSG_TRY(L->psi.alloc(ctx, sizeof(double) * (size_t)kd.n_terms * m->n_elems));
  MSG_CUDA(ctx, cudaMemcpyAsync(L->psi.ptr, kd.psi, sizeof(double) * (size_t)kd.n_terms * m->n_elems,
                                cudaMemcpyDeviceToDevice, ctx->stream));
  MSG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  L->kd = kd;
  L->kd.psi = L->psi.as<double>();
  MSG_TRY(L->d_xi.alloc(ctx, sizeof(double) * (size_t)Rp * kl->n_terms));
  MSG_TRY(L->d_slots.alloc(ctx, sizeof(int) * Rp));
  MSG_TRY(L->d_col.alloc(ctx, sizeof(double) * (size_t)std::max(1, m->n_dofs)));
  // the load (one vector for every request of the model)
  DevMem db;
  MSG_TRY(db.alloc(ctx, sizeof(double) * (size_t)std::max(1, m->n_dofs)));
  MSG_CUDA(ctx, cudaMemcpyAsync(db.ptr, b_host, sizeof(double) * m->n_dofs, cudaMemcpyHostToDevice, L->st));
  k_lattice_rhs<<<(m->n_dofs + 255) / 256, 256, 0, L->st>>>(m->n_dofs, m->d_pad_free_rows.as<int>(), db.as<double>(),
                                                            L->B.blat.as<double>());
  // every slot starts empty: scalars zero, done = 1 (not iterating)
  MSG_CUDA(ctx, cudaMemsetAsync(L->B.scal.ptr, 0, L->B.scal_bytes, L->st));
  k_fill_int<<<(Rp + 255) / 256, 256, 0, L->st>>>(L->B.s.done, Rp, 1);
  count_launch(ctx, 2);
  L->cfg = loop_cfg(ctx, &L->B, tol, 0);
  cudaGraphExec_t g = nullptr;
  MSG_TRY(block_graph(ctx, &L->B, L->cfg, &g));
  MSG_CUDA(ctx, cudaStreamSynchronize(L->st));
  *out = L.release();
  return MSG_OK;
}

void lane_destroy(Lane* L) { delete L; }
int lane_capacity(const Lane* L) { return L->capacity; }
int lane_n_dofs(const Lane* L) { return L->m->n_dofs; }
int lane_n_terms(const Lane* L) { return L->n_terms; }

// Queue request xi into `slot` (host side; initialised at the next cycle).
void lane_stage(Lane* L, int slot, const double* xi) {
  std::memcpy(L->h_xi + (size_t)L->n_pending * L->n_terms, xi, sizeof(double) * L->n_terms);
  L->h_slots[L->n_pending++] = slot;
}

// Stop a slot at the next cycle (its request was cancelled).
int lane_abort(Lane* L, int slot) {
  k_fill_int<<<1, 1, 0, L->st>>>(L->B.s.done + slot, 1, 1);
  return cudaGetLastError() == cudaSuccess ? MSG_OK : cuda_error(L->ctx, cudaGetLastError(), "lane abort");
}

// One boundary: start staged slots (zeroed vectors, field, Jacobi diagonal,
// norms), one FP64 true-residual step for every slot, then the next chunk of
// FP32 iterations (asynchronous). `state[slot]`: 0 iterating or empty, 1 converged,
// 2 breakdown, 3 iteration limit; its/res valid for finished slots.
int lane_cycle(Lane* L, int* state, int* its, double* res, int* n_active) {
  Context* ctx = L->ctx;
  BlockSys& B = L->B;
  cudaStream_t st = L->st;
  const int Rp = B.Rp;
  if (L->n_pending > 0) {
    const int n = L->n_pending;
    MSG_CUDA(ctx, cudaMemcpyAsync(L->d_xi.ptr, L->h_xi, sizeof(double) * (size_t)n * L->n_terms,
                                  cudaMemcpyHostToDevice, st));
    MSG_CUDA(ctx, cudaMemcpyAsync(L->d_slots.ptr, L->h_slots, sizeof(int) * n, cudaMemcpyHostToDevice, st));
    const size_t nrows = B.npad * 3;
    const int blocks = (int)std::min<size_t>((nrows * n + 255) / 256, (size_t)ctx->sm_count * 16);
    k_slot_reset<<<std::max(blocks, (n + 255) / 256), 256, 0, st>>>(
        n, L->d_slots.as<int>(), nrows, Rp, B.x.as<double>(), B.r32.as<float>(), B.rB.as<float>(), B.p.as<float>(),
        B.pB.as<float>(), B.q.as<float>(), B.qB.as<float>(), B.d.as<float>(), B.s);
    MSG_TRY(launch_kl_field_slots(st, L->m, &L->kd, n, L->d_slots.as<int>(), L->d_xi.as<double>(), Rp,
                                  B.E64.as<double>(), B.E32.as<float>()));
    k_dinv_slots<<<B.L.n_int, 128, 0, st>>>(B.L, B.kdiag, B.mdiag, B.E32.as<float>(), B.interior, n,
                                            L->d_slots.as<int>(), B.dinv.as<float>());
    count_launch(ctx, 3);
    gmg_fields(ctx, &B, st);
    MSG_TRY(block_bnorm(ctx, &B, B.blat.as<double>(), false));
    // the staging buffers are reused by the next cycle: wait for the copies
    MSG_CUDA(ctx, cudaStreamSynchronize(st));
    L->n_pending = 0;
  }
  MSG_TRY(block_update(ctx, &B, L->cfg, B.blat.as<double>(), false, L->tol, false, L->max_it));
  MSG_CUDA(ctx, cudaMemcpyAsync(L->h_flags, B.s.n_active, 36, cudaMemcpyDeviceToHost, st));
  MSG_CUDA(ctx, cudaMemcpyAsync(L->h_state, B.s.act, sizeof(int) * 5 * Rp, cudaMemcpyDeviceToHost, st));
  MSG_CUDA(ctx, cudaMemcpyAsync(L->h_res, B.s.res, sizeof(double) * Rp, cudaMemcpyDeviceToHost, st));
  MSG_CUDA(ctx, cudaStreamSynchronize(st));
  if (L->h_flags[8]) return set_error(ctx, MSG_ERR_TIMEOUT, "a bounded wait of the staged operator expired");
  const int* act = L->h_state;
  const int* done = L->h_state + Rp;
  const int* it = L->h_state + 2 * Rp;
  const int* brk = L->h_state + 3 * Rp;
  for (int r = 0; r < Rp; ++r) {
    state[r] = act[r] ? 0 : (brk[r] == 1 ? 2 : brk[r] == 2 ? 3 : (done[r] ? 1 : 0));
    its[r] = it[r];
    res[r] = L->h_res[r];
  }
  *n_active = L->h_flags[0];
  if (L->h_flags[0] > 0) {
    cudaGraphExec_t g = nullptr;
    MSG_TRY(block_graph(ctx, &B, L->cfg, &g));
    cudaError_t e = cudaGraphLaunch(g, st);
    if (e != cudaSuccess) return cuda_error(ctx, e, "lane chunk");
    count_launch(ctx, (B.gmg ? gmg_launches(&B) : 2) * L->cfg.chunk);
  }
  return MSG_OK;
}

// Displacements of a finished slot (DOF numbering) into the caller's host buffer.
int lane_fetch(Lane* L, int slot, double* X) {
  Context* ctx = L->ctx;
  const int nd = L->m->n_dofs;
  k_gather_column<<<(nd + 255) / 256, 256, 0, L->st>>>(nd, L->B.Rp, slot, L->m->d_pad_free_rows.as<int>(),
                                                      L->B.x.as<double>(), L->d_col.as<double>());
  count_launch(ctx);
  MSG_CUDA(ctx, cudaMemcpyAsync(L->h_col, L->d_col.ptr, sizeof(double) * nd, cudaMemcpyDeviceToHost, L->st));
  MSG_CUDA(ctx, cudaStreamSynchronize(L->st));
  if (X) std::memcpy(X, L->h_col, sizeof(double) * nd);
  return MSG_OK;
}

namespace {

// Node layout [(t * 3 + c) * Rp + r] (t: the node in generator order) to the
// padded lattice layout [(interior[t] * 3 + c) * Rp + r] and back; one CTA per
// node. Ghost nodes of the lattice are never written (they stay zero).
__global__ void k_node_to_lattice(int n_int, int Rp, const int* __restrict__ interior, const float* __restrict__ in,
                                  float* __restrict__ out) {
  const int t = blockIdx.x;
  if (t >= n_int) return;
  const size_t po = (size_t)interior[t] * 3 * Rp, no = (size_t)t * 3 * Rp;
  for (int i = threadIdx.x; i < 3 * Rp; i += blockDim.x) out[po + i] = in[no + i];
}

__global__ void k_lattice_to_node(int n_int, int Rp, const int* __restrict__ interior, const float* __restrict__ in,
                                  float* __restrict__ out) {
  const int t = blockIdx.x;
  if (t >= n_int) return;
  const size_t po = (size_t)interior[t] * 3 * Rp, no = (size_t)t * 3 * Rp;
  for (int i = threadIdx.x; i < 3 * Rp; i += blockDim.x) out[no + i] = in[po + i];
}

// The lattice batch of the preconditioner and the scalars its start pass
// reads: alpha = 0, so the start pass takes r' = r.
struct GmgPrecondImpl {
  BlockSys B;
  Scal s0;
  DevMem zero;
};

}  // namespace

int gmg_precond_create(Context* ctx, Mesh* lat, double nu, const MSG_KL* kl, const double* d_xi, int R, int Rp,
                       DevMem* own, void** out) {
  std::unique_ptr<GmgPrecondImpl> P(new GmgPrecondImpl());
  MSG_TRY(block_setup(ctx, lat, nu, 1.0, 1.0, 0.0, R, Rp, &P->B, own));
  if (!P->B.gmg)
    return set_error(ctx, MSG_ERR_NOT_STRUCTURED, "the lattice does not coarsen (or multigrid is off)");
  KLDevice kd;
  MSG_TRY(kl_prepare(ctx, lat, kl, &kd));
  MSG_TRY(block_field(ctx, lat, &P->B, &kd, d_xi));
  MSG_TRY(P->zero.alloc(ctx, sizeof(float) * Rp));
  MSG_CUDA(ctx, cudaMemsetAsync(P->zero.ptr, 0, sizeof(float) * Rp, ctx->stream));
  P->s0 = P->B.s;
  P->s0.alpha = P->zero.as<float>();
  MSG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  *out = P.release();
  return MSG_OK;
}

int gmg_precond_apply(Context* ctx, void* handle, const float* r_node, float* z_node, cudaStream_t st) {
  GmgPrecondImpl* P = static_cast<GmgPrecondImpl*>(handle);
  BlockSys& B = P->B;
  if (r_node) k_node_to_lattice<<<B.L.n_int, 256, 0, st>>>(B.L.n_int, B.Rp, B.interior, r_node, B.r32.as<float>());
  gmg_vcycle(&B, P->s0, true, st);
  if (z_node) k_lattice_to_node<<<B.L.n_int, 256, 0, st>>>(B.L.n_int, B.Rp, B.interior, B.qB.as<float>(), z_node);
  // the iteration's launches but beta, the direction pass and alpha
  count_launch(ctx, (r_node ? 1 : 0) + (z_node ? 1 : 0) + gmg_launches(&B) - 3);
  return MSG_OK;
}

void gmg_precond_buffers(void* handle, float** r_lat, float** z_lat, const int** node_to_lattice, int* Rp,
                         const double** zr_part, int* zr_blocks) {
  GmgPrecondImpl* P = static_cast<GmgPrecondImpl*>(handle);
  *r_lat = P->B.r32.as<float>();
  *z_lat = P->B.qB.as<float>();
  *node_to_lattice = P->B.interior;
  *Rp = P->B.Rp;
  // the level-0 post-sweep's partials z.r' ([tile][Rp][2], component 1)
  *zr_part = P->B.part_op.as<double>() + 1;
  *zr_blocks = P->B.pack ? P->B.n_tiles2 : P->B.n_tiles_m;
}

void gmg_precond_destroy(void* handle) { delete static_cast<GmgPrecondImpl*>(handle); }

}  // namespace msg
