// Host runtime of libmsolve_gpu.so: the extern "C" entry points of
// include/msolve_gpu.h, context and handle management, mesh analysis (3x3
// block sparsity pattern, assembly contribution map, structured-lattice
// detection) and the Monte Carlo batch driver.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>

#include "msg_internal.h"

namespace msg {

// ------------------------------------------------------------------ errors, memory
int set_error(Context* ctx, int code, const char* fmt, ...) {
  if (ctx) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    std::lock_guard<std::mutex> g(ctx->err_mu);
    ctx->last_error = buf;
  }
  return code;
}

int cuda_error(Context* ctx, cudaError_t e, const char* where) {
  const int code = (e == cudaErrorMemoryAllocation) ? MSG_ERR_OUT_OF_MEMORY : MSG_ERR_CUDA;
  return set_error(ctx, code, "CUDA error in %s: %s (%s)", where, cudaGetErrorName(e), cudaGetErrorString(e));
}

DevMem::~DevMem() { release(); }

void DevMem::release() {
  if (ptr) {
    cudaFree(ptr);
    if (ctx) ctx->used -= bytes;
  }
  ptr = nullptr;
  bytes = 0;
}

int DevMem::alloc(Context* c, size_t n) {
  release();
  ctx = c;
  if (n == 0) n = 16;
  if (c->budget && c->used + n > c->budget)
    return set_error(c, MSG_ERR_OUT_OF_MEMORY, "memory budget exceeded: %llu + %llu > %llu bytes",
                     (unsigned long long)c->used.load(), (unsigned long long)n, (unsigned long long)c->budget);
  cudaError_t e = cudaMalloc(&ptr, n);
  if (e != cudaSuccess) {
    ptr = nullptr;
    cudaGetLastError();
    if (e == cudaErrorMemoryAllocation)
      return set_error(c, MSG_ERR_OUT_OF_MEMORY, "device memory exhausted (cudaMalloc of %llu bytes)",
                       (unsigned long long)n);
    return cuda_error(c, e, "cudaMalloc");
  }
  bytes = n;
  c->used += n;
  return MSG_OK;
}

Matrix::~Matrix() {
  if (graph) cudaGraphExecDestroy(graph);
}

Context::~Context() {
  delete static_cast<msg_matrix*>(mc_matrix);
  delete mc_ke;
  delete mc_st;
  delete mc_E;
  for (auto& w : work) {
    delete w;
    w = nullptr;
  }
  for (DevMem* set : vc_pool) delete[] set;
  vc_pool.clear();
  for (LatticeRunner* r : lat_runners) delete r;
  lat_runners.clear();
  if (batch_graph) cudaGraphExecDestroy(batch_graph);
  for (auto& e : ev)
    if (e) cudaEventDestroy(e);
  if (copy_stream) {
    cudaStreamSynchronize(copy_stream);
    cudaStreamDestroy(copy_stream);
  }
  for (auto& e : pipe_ev)
    if (e) cudaEventDestroy(e);
  if (pipe_ready) cudaEventDestroy(pipe_ready);
  if (h_flags) cudaFreeHost(h_flags);
  if (h_stage) cudaFreeHost(h_stage);
}

int context_resources(Context* ctx) {
  if (!ctx->h_flags) {
    MSG_CUDA(ctx, cudaHostAlloc(&ctx->h_flags, 4096, cudaHostAllocMapped));
    MSG_CUDA(ctx, cudaHostGetDevicePointer(reinterpret_cast<void**>(&ctx->d_hflags), ctx->h_flags, 0));
  }
  if (!ctx->h_stage) MSG_CUDA(ctx, cudaMallocHost(&ctx->h_stage, 8192));
  for (auto& e : ctx->ev)
    if (!e) MSG_CUDA(ctx, cudaEventCreate(&e));
  return MSG_OK;
}

int pipe_flush(Context* ctx) {
  for (int i = 0; i < 2; ++i)
    if (ctx->pipe_pending[i]) {
      ctx->pipe_pending[i] = false;
      MSG_CUDA(ctx, cudaEventSynchronize(ctx->pipe_ev[i]));
    }
  return MSG_OK;
}

int workspace(Context* ctx, int slot, size_t bytes, void** out) {
  if (slot < 0 || slot >= kWorkSlots) return set_error(ctx, MSG_ERR_INVALID_ARGUMENT, "workspace slot");
  DevMem*& w = ctx->work[slot];
  if (!w) w = new DevMem();
  if (w->bytes < bytes) MSG_TRY(w->alloc(ctx, bytes));
  *out = w->ptr;
  return MSG_OK;
}

void retain(Context* ctx) { ctx->refs++; }

void release(Context* ctx) {
  if (--ctx->refs == 0) {
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    cudaStreamDestroy(ctx->stream);
    delete static_cast<msg_context*>(ctx);
  }
}

void retain(Mesh* m) { m->refs++; }

void release(Mesh* m) {
  if (--m->refs == 0) {
    Context* ctx = m->ctx;
    {
      std::lock_guard<std::recursive_mutex> lk(ctx->mu);
      cudaSetDevice(ctx->device);
      cudaStreamSynchronize(ctx->stream);
      if (ctx->mc_matrix && ctx->mc_matrix->mesh == m) {
        delete static_cast<msg_matrix*>(ctx->mc_matrix);
        ctx->mc_matrix = nullptr;
      }
      if (m->shadow) release(m->shadow);
      delete static_cast<msg_mesh*>(m);
    }
    release(ctx);
  }
}

template <class T>
static int upload(Context* ctx, DevMem& dst, const T* src, size_t n) {
  MSG_TRY(dst.alloc(ctx, sizeof(T) * n));
  if (n) MSG_CUDA(ctx, cudaMemcpyAsync(dst.ptr, src, sizeof(T) * n, cudaMemcpyHostToDevice, ctx->stream));
  return MSG_OK;
}

static bool cube_cached(Context* ctx, int kind, double h, double param, double* out) {
  std::lock_guard<std::mutex> g(ctx->cube_mu);
  for (const auto& c : ctx->cube_cache)
    if (c.kind == kind && c.h == h && c.param == param) {
      std::memcpy(out, c.v, sizeof(c.v));
      return true;
    }
  return false;
}

static void cube_store(Context* ctx, int kind, double h, double param, const double* v) {
  std::lock_guard<std::mutex> g(ctx->cube_mu);
  if (ctx->cube_cache.size() >= 32) ctx->cube_cache.erase(ctx->cube_cache.begin());
  Context::CubeMatrix c;
  c.kind = kind;
  c.h = h;
  c.param = param;
  std::memcpy(c.v, v, sizeof(c.v));
  ctx->cube_cache.push_back(c);
}

// Element stiffness of one cube of side h, E = 1, through the K1 kernel; full
// 24x24 (computed once per (h, nu) and context).
int unit_cube_khat(Context* ctx, double h, double nu, double* K576) {
  if (cube_cached(ctx, 0, h, nu, K576)) return MSG_OK;
  double xyz[24];
  for (int a = 0; a < 8; ++a) {
    const int ax = (a == 1 || a == 2 || a == 5 || a == 6), ay = (a == 2 || a == 3 || a == 6 || a == 7), az = a >= 4;
    xyz[3 * a] = ax * h; xyz[3 * a + 1] = ay * h; xyz[3 * a + 2] = az * h;
  }
  DevMem dx, dk, ds;
  MSG_TRY(upload(ctx, dx, xyz, 24));
  MSG_TRY(dk.alloc(ctx, sizeof(double) * 300));
  MSG_TRY(ds.alloc(ctx, sizeof(int)));
  MSG_CUDA(ctx, cudaMemsetAsync(ds.ptr, 0, sizeof(int), ctx->stream));
  MSG_TRY(launch_h8_ke(ctx, 1, dx.as<double>(), nullptr, 1.0, nu, dk.as<double>(), ds.as<int>()));
  double k300[300];
  MSG_CUDA(ctx, cudaMemcpyAsync(k300, dk.ptr, sizeof(k300), cudaMemcpyDeviceToHost, ctx->stream));
  MSG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  for (int i = 0; i < 24; ++i)
    for (int j = 0; j < 24; ++j) K576[i * 24 + j] = k300[packed_index(i, j)];
  for (int i = 1; i < 24; ++i)
    if (std::fabs(K576[i * 25] - K576[0]) > 1e-12 * std::fabs(K576[0]))
      return set_error(ctx, MSG_ERR_NOT_STRUCTURED, "cube stiffness has unequal diagonal entries");
  cube_store(ctx, 0, h, nu, K576);
  return MSG_OK;
}

int unit_cube_mhat(Context* ctx, double h, double rho, double* M576) {
  if (cube_cached(ctx, 1, h, rho, M576)) return MSG_OK;
  double xyz[24];
  for (int a = 0; a < 8; ++a) {
    const int ax = (a == 1 || a == 2 || a == 5 || a == 6), ay = (a == 2 || a == 3 || a == 6 || a == 7), az = a >= 4;
    xyz[3 * a] = ax * h; xyz[3 * a + 1] = ay * h; xyz[3 * a + 2] = az * h;
  }
  DevMem dx, dm, ds;
  MSG_TRY(upload(ctx, dx, xyz, 24));
  MSG_TRY(dm.alloc(ctx, sizeof(double) * 300));
  MSG_TRY(ds.alloc(ctx, sizeof(int)));
  MSG_CUDA(ctx, cudaMemsetAsync(ds.ptr, 0, sizeof(int), ctx->stream));
  MSG_TRY(launch_h8_me(ctx, 1, dx.as<double>(), rho, dm.as<double>(), ds.as<int>()));
  double m300[300];
  MSG_CUDA(ctx, cudaMemcpyAsync(m300, dm.ptr, sizeof(m300), cudaMemcpyDeviceToHost, ctx->stream));
  MSG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  for (int i = 0; i < 24; ++i)
    for (int j = 0; j < 24; ++j) M576[i * 24 + j] = m300[packed_index(i, j)];
  cube_store(ctx, 1, h, rho, M576);
  return MSG_OK;
}

// ------------------------------------------------------------------ mesh analysis
static int build_pattern(Mesh* m) {
  const int nn = m->n_nodes, ne = m->n_elems;
  // node adjacency through elements (CSR, sorted unique)
  std::vector<int64_t> cnt(nn + 1, 0);
  for (int e = 0; e < ne; ++e)
    for (int a = 0; a < 8; ++a) cnt[m->conn[8 * e + a] + 1] += 8;
  for (int i = 0; i < nn; ++i) cnt[i + 1] += cnt[i];
  std::vector<int> adj(cnt[nn]);
  std::vector<int64_t> fill(cnt.begin(), cnt.end() - 1);
  for (int e = 0; e < ne; ++e)
    for (int a = 0; a < 8; ++a)
      for (int b = 0; b < 8; ++b) adj[fill[m->conn[8 * e + a]]++] = m->conn[8 * e + b];
  std::vector<int> rowlen(nn);
  std::vector<int64_t> rowstart(nn);
  for (int i = 0; i < nn; ++i) {
    auto b = adj.begin() + cnt[i], en = adj.begin() + cnt[i + 1];
    std::sort(b, en);
    rowlen[i] = (int)(std::unique(b, en) - b);
    rowstart[i] = cnt[i];
  }
  BlockPattern& P = m->pat;
  P.n_rows = nn;
  P.n_slices = (nn + 31) / 32;
  P.slice_ptr.assign(P.n_slices + 1, 0);
  P.nnzb = 0;
  for (int z = 0; z < P.n_slices; ++z) {
    int w = 0;
    for (int l = 0; l < 32 && 32 * z + l < nn; ++l) w = std::max(w, rowlen[32 * z + l]);
    P.slice_ptr[z + 1] = P.slice_ptr[z] + w;
  }
  P.n_slots = P.slice_ptr[P.n_slices];
  P.col.assign(P.n_slots * 32, -1);
  P.diag_pos.assign(nn, -1);
  for (int row = 0; row < nn; ++row) {
    const int z = row / 32, lane = row % 32;
    for (int s = 0; s < rowlen[row]; ++s) {
      const int c = adj[rowstart[row] + s];
      const int64_t pos = (P.slice_ptr[z] + s) * 32 + lane;
      P.col[pos] = c;
      if (c == row) P.diag_pos[row] = (int)pos;
    }
    P.nnzb += rowlen[row];
  }
  // contribution lists in element order (deterministic summation order)
  const int64_t npos = P.n_slots * 32;
  P.contrib_ptr.assign(npos + 1, 0);
  std::vector<int64_t> where((size_t)ne * 64);
  for (int e = 0; e < ne; ++e)
    for (int a = 0; a < 8; ++a) {
      const int row = m->conn[8 * e + a];
      const int z = row / 32, lane = row % 32;
      const int* rb = adj.data() + rowstart[row];
      for (int b = 0; b < 8; ++b) {
        const int c = m->conn[8 * e + b];
        const int s = (int)(std::lower_bound(rb, rb + rowlen[row], c) - rb);
        const int64_t pos = (P.slice_ptr[z] + s) * 32 + lane;
        where[(size_t)e * 64 + a * 8 + b] = pos;
        P.contrib_ptr[pos + 1]++;
      }
    }
  for (int64_t p = 0; p < npos; ++p) P.contrib_ptr[p + 1] += P.contrib_ptr[p];
  P.contrib.assign(P.contrib_ptr[npos], 0);
  std::vector<int64_t> f2(P.contrib_ptr.begin(), P.contrib_ptr.end() - 1);
  for (int e = 0; e < ne; ++e)
    for (int ab = 0; ab < 64; ++ab) P.contrib[f2[where[(size_t)e * 64 + ab]]++] = e * 64 + ab;
  return MSG_OK;
}

// Structured cube lattice in generator order (Hexa8MeshGenerator.cs:508-568 node
// IDs x fastest, :1075-1089 element corners).
static void detect_structured(Mesh* m) {
  m->structured = false;
  const int nn = m->n_nodes, ne = m->n_elems;
  if (nn < 8 || ne < 1) return;
  const double* X = m->xyz.data();
  // axis extents from node 0 and the lattice size from the element count per axis
  double lo[3], hi[3];
  for (int a = 0; a < 3; ++a) { lo[a] = hi[a] = X[a]; }
  for (int i = 0; i < nn; ++i)
    for (int a = 0; a < 3; ++a) { lo[a] = std::min(lo[a], X[3 * i + a]); hi[a] = std::max(hi[a], X[3 * i + a]); }
  // element 0 edge length
  const int* c0 = m->conn.data();
  const double h = X[3 * c0[1]] - X[3 * c0[0]];
  if (!(h > 0)) return;
  int n[3];
  for (int a = 0; a < 3; ++a) {
    const double v = (hi[a] - lo[a]) / h;
    n[a] = (int)std::lround(v);
    if (n[a] < 1 || std::fabs(v - n[a]) > 1e-9 * std::max(1.0, v)) return;
  }
  const int NX = n[0] + 1, NY = n[1] + 1, NZ = n[2] + 1;
  if ((int64_t)NX * NY * NZ != nn || (int64_t)n[0] * n[1] * n[2] != ne) return;
  const double tol = 1e-9 * h;
  for (int k = 0, id = 0; k < NZ; ++k)
    for (int j = 0; j < NY; ++j)
      for (int i = 0; i < NX; ++i, ++id) {
        if (std::fabs(X[3 * id] - (lo[0] + i * h)) > tol || std::fabs(X[3 * id + 1] - (lo[1] + j * h)) > tol ||
            std::fabs(X[3 * id + 2] - (lo[2] + k * h)) > tol)
          return;
      }
  for (int k = 0, e = 0; k < n[2]; ++k)
    for (int j = 0; j < n[1]; ++j)
      for (int i = 0; i < n[0]; ++i, ++e) {
        const int b = i + NX * (j + NY * k);
        const int ref[8] = {b, b + 1, b + NX + 1, b + NX, b + NX * NY, b + NX * NY + 1, b + NX * NY + NX + 1,
                            b + NX * NY + NX};
        for (int a = 0; a < 8; ++a)
          if (m->conn[8 * e + a] != ref[a]) return;
      }
  m->structured = true;
  m->nx = n[0]; m->ny = n[1]; m->nz = n[2];
  m->h = h;
  for (int a = 0; a < 3; ++a) m->origin[a] = lo[a];
}

// Index maps of the padded lattice used by the batched matrix-free path.
// The generator's numbering and element order with any node coordinates
// (element 0 on node 0, x fastest; the cube test of detect_structured left out).
static void detect_lattice_topology(Mesh* m) {
  m->topo_lattice = false;
  const int nn = m->n_nodes, ne = m->n_elems;
  if (nn < 8 || ne < 1 || m->conn[0] != 0) return;
  const int NX = m->conn[3], NXY = m->conn[4];
  if (NX < 2 || NXY < 2 * NX || NXY % NX != 0 || nn % NXY != 0) return;
  const int nx = NX - 1, ny = NXY / NX - 1, nz = nn / NXY - 1;
  if (nz < 1 || (int64_t)nx * ny * nz != ne) return;
  for (int k = 0, e = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i, ++e) {
        const int b = i + NX * j + NXY * k;
        const int ref[8] = {b, b + 1, b + NX + 1, b + NX, b + NXY, b + NXY + 1, b + NXY + NX + 1, b + NXY + NX};
        for (int a = 0; a < 8; ++a)
          if (m->conn[8 * (size_t)e + a] != ref[a]) return;
      }
  m->topo_lattice = true;
  m->tnx = nx;
  m->tny = ny;
  m->tnz = nz;
}

static int build_padded_maps(Context* ctx, Mesh* m) {
  const int NX = m->nx + 1, NY = m->ny + 1, NZ = m->nz + 1;
  m->NXp = NX + 2; m->NYp = NY + 2; m->NZp = NZ + 2;
  const int64_t npad = (int64_t)m->NXp * m->NYp * m->NZp;
  if (npad * 3 > INT32_MAX) return set_error(ctx, MSG_ERR_INVALID_ARGUMENT, "lattice too large");
  auto pad = [&](int i, int j, int k) { return (i + 1) + m->NXp * ((j + 1) + m->NYp * (k + 1)); };
  std::vector<int> interior((size_t)NX * NY * NZ), elem_row(m->n_elems), rows(m->n_dofs);
  std::vector<uint8_t> pmask(npad, 7);
  for (int k = 0, t = 0; k < NZ; ++k)
    for (int j = 0; j < NY; ++j)
      for (int i = 0; i < NX; ++i, ++t) {
        const int p = pad(i, j, k);
        interior[t] = p;
        uint8_t mk = 0;
        for (int c = 0; c < 3; ++c) {
          const int d = m->dof[3 * (size_t)t + c];
          if (d < 0) mk |= (uint8_t)(1 << c);
          else rows[d] = 3 * p + c;
        }
        pmask[p] = mk;
      }
  for (int k = 0, e = 0; k < m->nz; ++k)
    for (int j = 0; j < m->ny; ++j)
      for (int i = 0; i < m->nx; ++i, ++e) elem_row[e] = pad(i, j, k);
  MSG_TRY(upload(ctx, m->d_pad_interior, interior.data(), interior.size()));
  MSG_TRY(upload(ctx, m->d_pad_elem_row, elem_row.data(), elem_row.size()));
  MSG_TRY(upload(ctx, m->d_pad_free_rows, rows.data(), rows.size()));
  MSG_TRY(upload(ctx, m->d_pad_mask, pmask.data(), pmask.size()));
  return MSG_OK;
}

static int create_mesh(Context* ctx, int n_nodes, const double* xyz, int n_elems, const int* conn, const int* dof,
                       int n_dofs, Mesh** out) {
  if (n_nodes <= 0 || n_elems <= 0 || !xyz || !conn || !dof || n_dofs < 0 || !out)
    return set_error(ctx, MSG_ERR_INVALID_ARGUMENT, "mesh: invalid sizes or null pointers");
  std::unique_ptr<msg_mesh> m(new msg_mesh());
  m->ctx = ctx;
  m->n_nodes = n_nodes; m->n_elems = n_elems; m->n_dofs = n_dofs;
  m->xyz.assign(xyz, xyz + 3 * (size_t)n_nodes);
  m->conn.assign(conn, conn + 8 * (size_t)n_elems);
  m->dof.assign(dof, dof + 3 * (size_t)n_nodes);
  for (size_t i = 0; i < m->conn.size(); ++i)
    if (m->conn[i] < 0 || m->conn[i] >= n_nodes)
      return set_error(ctx, MSG_ERR_INVALID_ARGUMENT, "mesh: element node index out of range");
  std::vector<int> free_rows(n_dofs, -1);
  std::vector<uint8_t> mask(n_nodes, 0);
  for (int i = 0; i < n_nodes; ++i)
    for (int c = 0; c < 3; ++c) {
      const int d = m->dof[3 * i + c];
      if (d == -1) { mask[i] |= (uint8_t)(1 << c); continue; }
      if (d < 0 || d >= n_dofs || free_rows[d] != -1)
        return set_error(ctx, MSG_ERR_INVALID_ARGUMENT, "mesh: DOF numbering is not a bijection onto 0..n_dofs-1");
      free_rows[d] = 3 * i + c;
    }
  for (int d = 0; d < n_dofs; ++d)
    if (free_rows[d] < 0) return set_error(ctx, MSG_ERR_INVALID_ARGUMENT, "mesh: DOF %d unused", d);
  MSG_TRY(build_pattern(m.get()));
  detect_structured(m.get());
  if (m->structured) MSG_TRY(build_padded_maps(ctx, m.get()));
  else detect_lattice_topology(m.get());
  std::vector<double> exyz(24 * (size_t)n_elems), cen(3 * (size_t)n_elems);
  for (int e = 0; e < n_elems; ++e) {
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (int a = 0; a < 8; ++a)
      for (int c = 0; c < 3; ++c) {
        const double v = m->xyz[3 * (size_t)m->conn[8 * e + a] + c];
        exyz[24 * (size_t)e + 3 * a + c] = v;
        lo[c] = std::min(lo[c], v);
        hi[c] = std::max(hi[c], v);
      }
    // Hexa8WithStochasticMaterial.GetStochasticPoints: min + extent/2
    for (int c = 0; c < 3; ++c) cen[3 * (size_t)e + c] = lo[c] + (hi[c] - lo[c]) / 2;
  }
  const BlockPattern& P = m->pat;
  MSG_TRY(upload(ctx, m->d_exyz, exyz.data(), exyz.size()));
  MSG_TRY(upload(ctx, m->d_centroid, cen.data(), cen.size()));
  MSG_TRY(upload(ctx, m->d_dof, m->dof.data(), m->dof.size()));
  MSG_TRY(upload(ctx, m->d_conn, m->conn.data(), m->conn.size()));
  MSG_TRY(upload(ctx, m->d_mask, mask.data(), mask.size()));
  MSG_TRY(upload(ctx, m->d_free_rows, free_rows.data(), free_rows.size()));
  MSG_TRY(upload(ctx, m->d_col, P.col.data(), P.col.size()));
  MSG_TRY(upload(ctx, m->d_slice_ptr, P.slice_ptr.data(), P.slice_ptr.size()));
  MSG_TRY(upload(ctx, m->d_contrib_ptr, P.contrib_ptr.data(), P.contrib_ptr.size()));
  MSG_TRY(upload(ctx, m->d_contrib, P.contrib.data(), P.contrib.size()));
  MSG_TRY(upload(ctx, m->d_diag_pos, P.diag_pos.data(), P.diag_pos.size()));
  MSG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  retain(ctx);
  *out = m.release();
  return MSG_OK;
}

static int assemble_from_device_ke(Context* ctx, Mesh* m, const double* d_Ke, Matrix* A) {
  if (!A->d_val.ptr) {
    MSG_TRY(A->d_val.alloc(ctx, sizeof(double) * (size_t)m->pat.n_slots * 32 * 9));
    MSG_TRY(A->d_dinv.alloc(ctx, sizeof(double) * (size_t)m->n_nodes * 3));
  }
  MSG_TRY(launch_bsr_assemble(ctx, m, d_Ke, A->d_val.as<double>()));
  MSG_TRY(launch_bsr_diag_inv(ctx, m, A->d_val.as<double>(), A->d_dinv.as<double>()));
  return MSG_OK;
}

// Element matrices for per-element E (device), then assembly into A.
static int assemble_from_device_E(Context* ctx, Mesh* m, const double* d_E, double nu, Matrix* A, DevMem& ke,
                                  DevMem& st, int* neg_det) {
  // ke may be a buffer kept from a call on another mesh: grow it to this mesh
  const size_t ke_bytes = sizeof(double) * 300 * (size_t)m->n_elems;
  if (!ke.ptr || ke.bytes < ke_bytes) MSG_TRY(ke.alloc(ctx, ke_bytes));
  if (!st.ptr) MSG_TRY(st.alloc(ctx, sizeof(int)));
  MSG_CUDA(ctx, cudaMemsetAsync(st.ptr, 0, sizeof(int), ctx->stream));
  MSG_TRY(launch_h8_ke(ctx, m->n_elems, m->d_exyz.as<double>(), d_E, 0.0, nu, ke.as<double>(), st.as<int>()));
  MSG_TRY(assemble_from_device_ke(ctx, m, ke.as<double>(), A));
  if (neg_det) {
    MSG_CUDA(ctx, cudaMemcpyAsync(neg_det, st.ptr, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    MSG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  }
  return MSG_OK;
}

// Monte Carlo batch, device inputs.
static int mc_batch(Context* ctx, Mesh* m, double nu, const MSG_KL* kl, int R, const double* d_xi, const double* d_b,
                    int mode, int max_it, double tol, int tip_dof, double* d_X, double* tip, int* iterations,
                    double* rel_res) {
  NvtxRange range("msg: Monte Carlo batch");
  if (R <= 0 || !kl || !d_xi || !d_b || max_it <= 0 || !(tol > 0))
    return set_error(ctx, MSG_ERR_INVALID_ARGUMENT, "MC batch: invalid arguments");
  if (tip_dof >= m->n_dofs) return set_error(ctx, MSG_ERR_INVALID_ARGUMENT, "tip_dof out of range");
  // realizations padded to 64: the packed level operator works on pairs of 32-wide groups
  const int Rp = (R + 63) / 64 * 64;
  MSG_TRY(context_resources(ctx));
  cudaEvent_t e0 = ctx->ev[8], e1 = ctx->ev[9];
  cudaEventRecord(e0, ctx->stream);
  KLDevice kd;
  MSG_TRY(kl_prepare(ctx, m, kl, &kd));
  int status = MSG_OK;
  // meshes that are not cube lattices (distorted or unstructured): the mixed mode
  // solves every realization at once element by element (element_batch = 1), or
  // realization by realization with the assembled FP32-value PCG and FP64
  // refinement (MSG_PCG_SOLVE_MIXED's loop, element_batch = 0), to the same FP64
  // true residual
  const bool mixed_general = mode == MSG_MODE_MIXED_BATCHED && !m->structured;
  const bool per_realization = mode == MSG_MODE_FP64_BSR || (mixed_general && !ctx->element_batch);
  if (mixed_general && ctx->element_batch) {
    std::vector<RgInput> in(1);
    in[0].m = m;
    in[0].nu = nu;
    in[0].kl = kl;
    in[0].R = R;
    in[0].d_xi = d_xi;
    in[0].d_b = d_b;
    in[0].d_X = d_X;
    in[0].h_tip = tip;
    in[0].tip_dof = tip_dof;
    in[0].h_its = iterations;
    in[0].h_res = rel_res;
    status = ebe_solve(ctx, in, max_it, tol);
  } else if (mode == MSG_MODE_MIXED_BATCHED && m->structured) {
    BatchOut o;
    std::vector<double> htip(R);
    o.tip = tip ? htip.data() : nullptr;
    o.iterations = iterations;
    o.rel_res = rel_res;
    status = block_mixed_solve(ctx, m, nu, &kd, d_xi, R, Rp, d_b, max_it, tol, tip_dof, d_X, o);
    if (tip) std::copy(htip.begin(), htip.end(), tip);
  } else if (per_realization) {
    const bool mixed = mode == MSG_MODE_MIXED_BATCHED;
    // the assembled matrix and its buffers stay in the context for the next call on this mesh
    if (ctx->mc_matrix && ctx->mc_matrix->mesh != m) {
      delete static_cast<msg_matrix*>(ctx->mc_matrix);
      ctx->mc_matrix = nullptr;
    }
    if (!ctx->mc_matrix) {
      ctx->mc_matrix = new msg_matrix();
      ctx->mc_matrix->mesh = m;  // weak: release(Mesh*) drops this matrix with its mesh
    }
    if (!ctx->mc_ke) ctx->mc_ke = new DevMem();
    if (!ctx->mc_st) ctx->mc_st = new DevMem();
    if (!ctx->mc_E) ctx->mc_E = new DevMem();
    Matrix* A = ctx->mc_matrix;
    const size_t eb = sizeof(double) * (size_t)m->n_elems * R;
    if (ctx->mc_E->bytes < eb) {
      ctx->mc_E->release();
      MSG_TRY(ctx->mc_E->alloc(ctx, eb));
    }
    MSG_TRY(launch_kl_field(ctx, m, &kd, R, Rp, d_xi, nullptr, nullptr, ctx->mc_E->as<double>()));
    const size_t n3 = 3 * (size_t)m->n_nodes;
    if (!A->d_bn.ptr) {
      MSG_TRY(A->d_bd.alloc(ctx, sizeof(double) * std::max(1, m->n_dofs)));
      MSG_TRY(A->d_bn.alloc(ctx, sizeof(double) * n3));
      MSG_TRY(A->d_xn.alloc(ctx, sizeof(double) * n3));
    }
    MSG_CUDA(ctx, cudaMemsetAsync(A->d_bn.ptr, 0, sizeof(double) * n3, ctx->stream));
    MSG_TRY(launch_dof_to_node(ctx, m, d_b, A->d_bn.as<double>(), 1, 0, 0));
    for (int r = 0; r < R; ++r) {
      MSG_TRY(assemble_from_device_E(ctx, m, ctx->mc_E->as<double>() + (size_t)r * m->n_elems, nu, A, *ctx->mc_ke,
                                     *ctx->mc_st, nullptr));
      int its = 0, pst = 0;
      double rr = 0;
      if (mixed && A->d_val32.ptr) {  // the FP32 copy of this realization's values
        const size_t nv = (size_t)m->pat.n_slots * 32 * 9;
        MSG_TRY(launch_to_f32(ctx, nv, A->d_val.as<double>(), A->d_val32.as<float>()));
      }
      MSG_TRY(pcg_solve_device(ctx, A, A->d_bn.as<double>(), A->d_xn.as<double>(), max_it, tol, &its, &rr, &pst,
                               mixed));
      double* xout = d_X ? d_X + (size_t)r * m->n_dofs : A->d_bd.as<double>();
      MSG_TRY(launch_node_to_dof(ctx, m, A->d_xn.as<double>(), xout, 1, 0, 0));
      if (tip && tip_dof >= 0) {
        MSG_CUDA(ctx, cudaMemcpyAsync(tip + r, xout + tip_dof, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
      }
      if (iterations) iterations[r] = its + (pst == MSG_OK ? 1 : 0);  // matrix products
      if (rel_res) rel_res[r] = rr;
      if (pst != MSG_OK && status == MSG_OK) status = pst;
    }
    MSG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (status != MSG_OK)
      set_error(ctx, status, mixed ? "mixed batch: a realization did not converge" : "FP64 batch: a realization did not converge");
  } else {
    return set_error(ctx, MSG_ERR_INVALID_ARGUMENT, "unknown mode %d", mode);
  }
  cudaEventRecord(e1, ctx->stream);
  cudaEventSynchronize(e1);
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  ctx->t_phase[4] = ms;
  return status;
}

// KL 1-D eigen-pairs of exp(-|x-y|/l) on [-A, A]: roots of
// c cos(wA) - w sin(wA) (cos modes, odd index) and w cos(wA) + c sin(wA) (sin
// modes, even index), c = 1/l, by safeguarded Newton inside the bracket.
static double kl_root(double A, double c, bool is_sin, double lo, double hi) {
  auto f = [&](double w) { return is_sin ? w * std::cos(w * A) + c * std::sin(w * A) : c * std::cos(w * A) - w * std::sin(w * A); };
  auto df = [&](double w) {
    return is_sin ? std::cos(w * A) - w * A * std::sin(w * A) + c * A * std::cos(w * A)
                  : -c * A * std::sin(w * A) - std::sin(w * A) - w * A * std::cos(w * A);
  };
  double flo = f(lo);
  double w = 0.5 * (lo + hi);
  for (int it = 0; it < 200; ++it) {
    const double fw = f(w);
    if (fw == 0) return w;
    if ((fw > 0) == (flo > 0)) { lo = w; flo = fw; } else { hi = w; }
    const double d = df(w);
    double wn = (d != 0) ? w - fw / d : 0.5 * (lo + hi);
    if (!(wn > lo && wn < hi)) wn = 0.5 * (lo + hi);
    if (std::fabs(wn - w) <= 1e-16 * std::fabs(w) || hi - lo <= 4e-16 * hi) { w = wn; break; }
    w = wn;
  }
  return w;
}

int lattice_shadow(Context* ctx, Mesh* m, Mesh** out) {
  if (m->structured) {  // a cube lattice is its own
    *out = m;
    return MSG_OK;
  }
  std::lock_guard<std::mutex> lock(m->shadow_mu);
  if (!m->topo_lattice) return set_error(ctx, MSG_ERR_NOT_STRUCTURED, "mesh has no lattice topology");
  if (!m->shadow) {
    // cubes of the mean spacing of the mesh's bounding box, from its lower corner
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (int i = 0; i < m->n_nodes; ++i)
      for (int a = 0; a < 3; ++a) {
        lo[a] = std::min(lo[a], m->xyz[3 * (size_t)i + a]);
        hi[a] = std::max(hi[a], m->xyz[3 * (size_t)i + a]);
      }
    const int n[3] = {m->tnx, m->tny, m->tnz};
    double h = 0.0;
    for (int a = 0; a < 3; ++a) h += (hi[a] - lo[a]) / n[a] / 3.0;
    if (!(h > 0)) return set_error(ctx, MSG_ERR_NOT_STRUCTURED, "degenerate lattice extent");
    std::vector<double> xyz(3 * (size_t)m->n_nodes);
    for (int k = 0, t = 0; k <= n[2]; ++k)
      for (int j = 0; j <= n[1]; ++j)
        for (int i = 0; i <= n[0]; ++i, ++t) {
          xyz[3 * (size_t)t] = lo[0] + i * h;
          xyz[3 * (size_t)t + 1] = lo[1] + j * h;
          xyz[3 * (size_t)t + 2] = lo[2] + k * h;
        }
    Mesh* sh = nullptr;
    MSG_TRY(create_mesh(ctx, m->n_nodes, xyz.data(), m->n_elems, m->conn.data(), m->dof.data(), m->n_dofs, &sh));
    if (!sh->structured) {
      release(sh);
      return set_error(ctx, MSG_ERR_NOT_STRUCTURED, "lattice shadow was not recognised as a cube lattice");
    }
    m->shadow = sh;
  }
  *out = m->shadow;
  return MSG_OK;
}

}  // namespace msg

using namespace msg;

#define CTX_GUARD(ctx)                                        \
  if (!(ctx)) return MSG_ERR_INVALID_ARGUMENT;                \
  std::lock_guard<std::recursive_mutex> _lk((ctx)->mu);       \
  cudaSetDevice((ctx)->device)

extern "C" {

int MSG_VERSION(void) { return 100; }

int MSG_CREATE(int device, uint64_t mem_budget_bytes, MSG_CTX* out) {
  if (!out) return MSG_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) { cudaGetLastError(); return MSG_ERR_NO_DEVICE; }
  if (device < 0 || device >= n) return MSG_ERR_INVALID_ARGUMENT;
  std::unique_ptr<msg_context> c(new msg_context());
  c->device = device;
  c->budget = mem_budget_bytes;
  if (cudaSetDevice(device) != cudaSuccess) return MSG_ERR_CUDA;
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) return MSG_ERR_CUDA;
  cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, device);
  // MSG_PCG_SOLVE_NOALLOC's scratch array: its device address is resolved here,
  // outside any solve (the lookup may load the module and create the array)
  if (noalloc_scratch_address(&c->noalloc_scratch) != cudaSuccess) { cudaGetLastError(); return MSG_ERR_CUDA; }
  *out = c.release();
  return MSG_OK;
}

int MSG_DESTROY(MSG_CTX ctx) {
  if (!ctx) return MSG_ERR_INVALID_ARGUMENT;
  {
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    if (ctx->server) server_destroy(ctx);  // the serving lanes hold meshes of this context
    pipe_flush(ctx);                       // pipelined copies to the caller's X
  }
  release(ctx);  // freed once the last mesh/matrix of this context is destroyed
  return MSG_OK;
}

const char* MSG_LAST_ERROR(MSG_CTX ctx) { return ctx ? ctx->last_error.c_str() : "null context"; }

int MSG_SET_OPTION(MSG_CTX ctx, const char* key, double value) {
  CTX_GUARD(ctx);
  if (!key) return set_error(ctx, MSG_ERR_INVALID_ARGUMENT, "null option key");
  if (!std::strcmp(key, "reliable_delta") && value > 0 && value < 1) { ctx->reliable_delta = value; return MSG_OK; }
  if (!std::strcmp(key, "chunk") && value >= 2 && value <= 256) { ctx->chunk = ((int)value) & ~1; return MSG_OK; }
  if (!std::strcmp(key, "fixed_updates") && (value == 0 || value == 1)) { ctx->fixed_updates = (int)value; return MSG_OK; }
  if (!std::strcmp(key, "multigrid") && (value == 0 || value == 1 || value == 2)) {
    ctx->multigrid = (int)value;
    return MSG_OK;
  }
  if (!std::strcmp(key, "multigrid_levels") && value >= 2 && value <= kGmgMaxLevels && value == (int)value) {
    ctx->mg_levels = (int)value;
    return MSG_OK;
  }
  if (!std::strcmp(key, "multigrid_sweeps") && value >= 1 && value <= 1000 && value == (int)value) {
    ctx->mg_sweeps = (int)value;
    return MSG_OK;
  }
  if (!std::strcmp(key, "multigrid_omega") && value >= 0 && value < 1) { ctx->mg_omega = value; return MSG_OK; }
  if (!std::strcmp(key, "multigrid_delta") && value > 0 && value < 1) { ctx->mg_delta = value; return MSG_OK; }
  if (!std::strcmp(key, "multigrid_packed") && (value == 0 || value == 1)) { ctx->mg_packed = (int)value; return MSG_OK; }
  if (!std::strcmp(key, "tensor_operator") && (value == 0 || value == 1)) { ctx->tensor_op = (int)value; return MSG_OK; }
  if (!std::strcmp(key, "spmv32_shape") && value >= 0 && value <= 3 && value == (int)value) {
    ctx->spmv32_shape = (int)value;
    return MSG_OK;
  }
  if (!std::strcmp(key, "element_batch") && (value == 0 || value == 1)) {
    ctx->element_batch = (int)value;
    return MSG_OK;
  }
  if (!std::strcmp(key, "element_groups") && (value == 0 || value == 1 || value == 2 || value == 4 || value == 8)) {
    ctx->element_groups = (int)value;
    return MSG_OK;
  }
  if (!std::strcmp(key, "ragged_lattice_loop") && (value == 0 || value == 1)) {
    ctx->ragged_lattice_loop = (int)value;
    return MSG_OK;
  }
  if (!std::strcmp(key, "ragged_side_by_side") && (value == 0 || value == 1)) {
    ctx->ragged_side_by_side = (int)value;
    return MSG_OK;
  }
  if (!std::strcmp(key, "newmark_predictor") && (value == 0 || value == 1)) {
    ctx->nm_predictor = (int)value;
    return MSG_OK;
  }
  if (!std::strcmp(key, "multigrid_fused_coarse") && (value == 0 || value == 1)) {
    ctx->mg_fused_coarse = (int)value;
    return MSG_OK;
  }
  if (!std::strcmp(key, "serve_persistent") && (value == 0 || value == 1)) {
    ctx->serve_persistent = (int)value;
    return MSG_OK;
  }
  if (!std::strcmp(key, "serve_priority") && (value == 0 || value == 1)) {
    ctx->serve_priority = (int)value;
    return MSG_OK;
  }
  return set_error(ctx, MSG_ERR_INVALID_ARGUMENT, "unknown option or value out of range: %s", key);
}

int MSG_GET_OPTION(MSG_CTX ctx, const char* key, double* value) {
  CTX_GUARD(ctx);
  if (!key || !value) return set_error(ctx, MSG_ERR_INVALID_ARGUMENT, "null option key or value");
  if (!std::strcmp(key, "device_free_memory")) {  // read-only: free bytes on the context's device
    size_t free_b = 0, total_b = 0;
    MSG_CUDA(ctx, cudaSetDevice(ctx->device));
    MSG_CUDA(ctx, cudaMemGetInfo(&free_b, &total_b));
    *value = (double)free_b;
    return MSG_OK;
  }
  const struct {
    const char* name;
    double v;
  } opts[] = {{"reliable_delta", ctx->reliable_delta},
              {"chunk", (double)ctx->chunk},
              {"fixed_updates", (double)ctx->fixed_updates},
              {"multigrid", (double)ctx->multigrid},
              {"multigrid_levels", (double)ctx->mg_levels},
              {"multigrid_sweeps", (double)ctx->mg_sweeps},
              {"multigrid_omega", ctx->mg_omega},
              {"multigrid_delta", ctx->mg_delta},
              {"multigrid_packed", (double)ctx->mg_packed},
              {"tensor_operator", (double)ctx->tensor_op},
              {"spmv32_shape", (double)ctx->spmv32_shape},
              {"element_batch", (double)ctx->element_batch},
              {"element_groups", (double)ctx->element_groups},
              {"ragged_lattice_loop", (double)ctx->ragged_lattice_loop},
              {"ragged_side_by_side", (double)ctx->ragged_side_by_side},
              {"newmark_predictor", (double)ctx->nm_predictor},
              {"multigrid_fused_coarse", (double)ctx->mg_fused_coarse},
              {"serve_persistent", (double)ctx->serve_persistent},
              {"serve_priority", (double)ctx->serve_priority},
              // read-only: device memory charged to the context and its budget (bytes)
              {"memory_used", (double)ctx->used.load()},
              {"memory_budget", (double)ctx->budget}};
  for (const auto& o : opts)
    if (!std::strcmp(key, o.name)) {
      *value = o.v;
      return MSG_OK;
    }
  return set_error(ctx, MSG_ERR_INVALID_ARGUMENT, "unknown option: %s", key);
}

int MSG_STATS(MSG_CTX ctx, int64_t* launches, double* t8) {
  if (!ctx) return MSG_ERR_INVALID_ARGUMENT;
  if (launches) *launches = ctx->launches.load();
  if (t8) {
    for (int i = 0; i < 5; ++i) t8[i] = ctx->t_phase[i];
    const double n = (double)ctx->op_samples;
    t8[5] = n > 0 ? ctx->op_ms_sum / n : 0.0;
    t8[6] = n > 0 ? ctx->upd_ms_sum / n : 0.0;
    t8[7] = n;
  }
  return MSG_OK;
}

int MSG_STATS_RESET(MSG_CTX ctx) {
  if (!ctx) return MSG_ERR_INVALID_ARGUMENT;
  ctx->op_ms_sum = ctx->upd_ms_sum = 0;
  ctx->op_samples = 0;
  return MSG_OK;
}

int MSG_WAIT_SELFTEST(MSG_CTX ctx, int64_t polls) {
  CTX_GUARD(ctx);
  if (polls < 1 || polls > (int64_t)1 << 24)
    return set_error(ctx, MSG_ERR_INVALID_ARGUMENT, "wait self-test: polls must be in [1, 2^24]");
  int expired = 0;
  MSG_TRY(wait_selftest(ctx, (long)polls, &expired));
  return expired ? set_error(ctx, MSG_ERR_TIMEOUT, "bounded wait expired (self-test)") : MSG_OK;
}

int MSG_H8_KE_BATCH(MSG_CTX ctx, int n, const double* xyz, const double* E, double nu, double* Ke) {
  CTX_GUARD(ctx);
  if (n < 0 || (n > 0 && (!xyz || !E || !Ke))) return set_error(ctx, MSG_ERR_INVALID_ARGUMENT, "KE batch: bad args");
  if (n == 0) return MSG_OK;
  if (!(nu > -1.0 && nu < 0.5)) return set_error(ctx, MSG_ERR_INVALID_ARGUMENT, "Poisson ratio out of (-1, 0.5)");
  DevMem dx, dE, dK, ds;
  MSG_TRY(upload(ctx, dx, xyz, 24 * (size_t)n));
  MSG_TRY(upload(ctx, dE, E, (size_t)n));
  MSG_TRY(dK.alloc(ctx, sizeof(double) * 300 * (size_t)n));
  MSG_TRY(ds.alloc(ctx, sizeof(int)));
  MSG_CUDA(ctx, cudaMemsetAsync(ds.ptr, 0, sizeof(int), ctx->stream));
  MSG_TRY(launch_h8_ke(ctx, n, dx.as<double>(), dE.as<double>(), 0.0, nu, dK.as<double>(), ds.as<int>()));
  int st = 0;
  MSG_CUDA(ctx, cudaMemcpyAsync(Ke, dK.ptr, sizeof(double) * 300 * (size_t)n, cudaMemcpyDeviceToHost, ctx->stream));
  MSG_CUDA(ctx, cudaMemcpyAsync(&st, ds.ptr, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  MSG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  if (st != 0) return set_error(ctx, st, "negative or tiny Jacobian determinant (H8)");
  return MSG_OK;
}

int MSG_H8_ME_BATCH(MSG_CTX ctx, int n, const double* xyz, double rho, double* Me) {
  CTX_GUARD(ctx);
  if (n < 0 || (n > 0 && (!xyz || !Me))) return set_error(ctx, MSG_ERR_INVALID_ARGUMENT, "ME batch: bad args");
  if (n == 0) return MSG_OK;
  DevMem dx, dM, ds;
  MSG_TRY(upload(ctx, dx, xyz, 24 * (size_t)n));
  MSG_TRY(dM.alloc(ctx, sizeof(double) * 300 * (size_t)n));
  MSG_TRY(ds.alloc(ctx, sizeof(int)));
  MSG_CUDA(ctx, cudaMemsetAsync(ds.ptr, 0, sizeof(int), ctx->stream));
  MSG_TRY(launch_h8_me(ctx, n, dx.as<double>(), rho, dM.as<double>(), ds.as<int>()));
  int st = 0;
  MSG_CUDA(ctx, cudaMemcpyAsync(Me, dM.ptr, sizeof(double) * 300 * (size_t)n, cudaMemcpyDeviceToHost, ctx->stream));
  MSG_CUDA(ctx, cudaMemcpyAsync(&st, ds.ptr, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  MSG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  if (st != 0) return set_error(ctx, st, "negative or tiny Jacobian determinant (H8)");
  return MSG_OK;
}

int MSG_H8_STRESS_BATCH(MSG_CTX ctx, int n, const double* xyz, const double* E, double nu, const double* u,
                        const double* du, double* strains, double* stresses, double* forces) {
  CTX_GUARD(ctx);
  if (n < 0 || (n > 0 && (!xyz || !E || !u))) return set_error(ctx, MSG_ERR_INVALID_ARGUMENT, "stress batch: bad args");
  if (n == 0) return MSG_OK;
  if (!(nu > -1.0 && nu < 0.5)) return set_error(ctx, MSG_ERR_INVALID_ARGUMENT, "Poisson ratio out of (-1, 0.5)");
  DevMem dx, dE, du_, ddu, dS, dT, dF, ds;
  MSG_TRY(upload(ctx, dx, xyz, 24 * (size_t)n));
  MSG_TRY(upload(ctx, dE, E, (size_t)n));
  MSG_TRY(upload(ctx, du_, u, 24 * (size_t)n));
  if (du) MSG_TRY(upload(ctx, ddu, du, 24 * (size_t)n));
  if (strains) MSG_TRY(dS.alloc(ctx, sizeof(double) * 48 * (size_t)n));
  if (stresses) MSG_TRY(dT.alloc(ctx, sizeof(double) * 48 * (size_t)n));
  if (forces) MSG_TRY(dF.alloc(ctx, sizeof(double) * 24 * (size_t)n));
  MSG_TRY(ds.alloc(ctx, sizeof(int)));
  MSG_CUDA(ctx, cudaMemsetAsync(ds.ptr, 0, sizeof(int), ctx->stream));
  MSG_TRY(launch_h8_stress(ctx, n, dx.as<double>(), dE.as<double>(), 0.0, nu, du_.as<double>(),
                           du ? ddu.as<double>() : nullptr, nullptr, nullptr, nullptr, n, 0, dS.as<double>(),
                           dT.as<double>(), dF.as<double>(), ds.as<int>()));
  int st = 0;
  if (strains)
    MSG_CUDA(ctx, cudaMemcpyAsync(strains, dS.ptr, sizeof(double) * 48 * (size_t)n, cudaMemcpyDeviceToHost, ctx->stream));
  if (stresses)
    MSG_CUDA(ctx, cudaMemcpyAsync(stresses, dT.ptr, sizeof(double) * 48 * (size_t)n, cudaMemcpyDeviceToHost,
                                  ctx->stream));
  if (forces)
    MSG_CUDA(ctx, cudaMemcpyAsync(forces, dF.ptr, sizeof(double) * 24 * (size_t)n, cudaMemcpyDeviceToHost, ctx->stream));
  MSG_CUDA(ctx, cudaMemcpyAsync(&st, ds.ptr, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  MSG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  if (st != 0) return set_error(ctx, st, "negative or tiny Jacobian determinant (H8)");
  return MSG_OK;
}

int MSG_STRESS_BATCH_DEVICE(MSG_MESH mesh, int R, const double* E_dev, double nu, const double* X_dev,
                            double* strains_dev, double* stresses_dev, double* forces_dev) {
  if (!mesh) return MSG_ERR_INVALID_ARGUMENT;
  Context* ctx = mesh->ctx;
  CTX_GUARD(ctx);
  if (R < 0 || (R > 0 && (!E_dev || !X_dev)))
    return set_error(ctx, MSG_ERR_INVALID_ARGUMENT, "stress batch: bad args");
  if (R == 0) return MSG_OK;
  if (!(nu > -1.0 && nu < 0.5)) return set_error(ctx, MSG_ERR_INVALID_ARGUMENT, "Poisson ratio out of (-1, 0.5)");
  const int64_t n = (int64_t)R * mesh->n_elems;
  if (n > INT32_MAX) return set_error(ctx, MSG_ERR_INVALID_ARGUMENT, "stress batch: R * n_elems too large");
  DevMem ds;
  MSG_TRY(ds.alloc(ctx, sizeof(int)));
  MSG_CUDA(ctx, cudaMemsetAsync(ds.ptr, 0, sizeof(int), ctx->stream));
  MSG_TRY(launch_h8_stress(ctx, (int)n, mesh->d_exyz.as<double>(), E_dev, 0.0, nu, nullptr, nullptr, X_dev,
                           mesh->d_conn.as<int>(), mesh->d_dof.as<int>(), mesh->n_elems, mesh->n_dofs, strains_dev,
                           stresses_dev, forces_dev, ds.as<int>()));
  int st = 0;
  MSG_CUDA(ctx, cudaMemcpyAsync(&st, ds.ptr, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  MSG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  if (st != 0) return set_error(ctx, st, "negative or tiny Jacobian determinant (H8)");
  return MSG_OK;
}

int MSG_MESH_CREATE(MSG_CTX ctx, int n_nodes, const double* xyz, int n_elems, const int* conn, const int* dof,
                    int n_dofs, MSG_MESH* out) {
  CTX_GUARD(ctx);
  Mesh* m = nullptr;
  MSG_TRY(create_mesh(ctx, n_nodes, xyz, n_elems, conn, dof, n_dofs, &m));
  *out = static_cast<msg_mesh*>(m);
  return MSG_OK;
}

int MSG_MESH_INFO(MSG_MESH m, int64_t* info) {
  if (!m || !info) return MSG_ERR_INVALID_ARGUMENT;
  info[0] = m->structured; info[1] = m->nx; info[2] = m->ny; info[3] = m->nz;
  info[4] = m->n_dofs; info[5] = m->pat.n_rows; info[6] = m->pat.nnzb; info[7] = m->n_elems;
  return MSG_OK;
}

int MSG_MESH_DESTROY(MSG_MESH m) {
  if (!m) return MSG_ERR_INVALID_ARGUMENT;
  release(static_cast<Mesh*>(m));
  return MSG_OK;
}

int MSG_ASSEMBLE_BSR(MSG_MESH m, const double* E, double nu, MSG_MAT* out) {
  if (!m || !E || !out) return MSG_ERR_INVALID_ARGUMENT;
  Context* ctx = m->ctx;
  CTX_GUARD(ctx);
  if (!(nu > -1.0 && nu < 0.5)) return set_error(ctx, MSG_ERR_INVALID_ARGUMENT, "Poisson ratio out of (-1, 0.5)");
  std::unique_ptr<msg_matrix> A(new msg_matrix());
  A->mesh = m;
  DevMem dE, ke, st;
  MSG_TRY(upload(ctx, dE, E, (size_t)m->n_elems));
  int neg = 0;
  MSG_TRY(assemble_from_device_E(ctx, m, dE.as<double>(), nu, A.get(), ke, st, &neg));
  if (neg != 0) return set_error(ctx, neg, "negative or tiny Jacobian determinant (H8)");
  retain(static_cast<Mesh*>(m));
  *out = A.release();
  return MSG_OK;
}

int MSG_ASSEMBLE_BSR_KE(MSG_MESH m, const double* Ke, MSG_MAT* out) {
  if (!m || !Ke || !out) return MSG_ERR_INVALID_ARGUMENT;
  Context* ctx = m->ctx;
  CTX_GUARD(ctx);
  std::unique_ptr<msg_matrix> A(new msg_matrix());
  A->mesh = m;
  DevMem dK;
  MSG_TRY(upload(ctx, dK, Ke, 300 * (size_t)m->n_elems));
  MSG_TRY(assemble_from_device_ke(ctx, m, dK.as<double>(), A.get()));
  MSG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  retain(static_cast<Mesh*>(m));
  *out = A.release();
  return MSG_OK;
}

int MSG_MAT_MULTIPLY(MSG_MAT A, const double* x, double* y) {
  if (!A || !x || !y) return MSG_ERR_INVALID_ARGUMENT;
  Mesh* m = A->mesh;
  Context* ctx = m->ctx;
  CTX_GUARD(ctx);
  const size_t n3 = 3 * (size_t)m->n_nodes;
  DevMem dxd, dxn, dyn, dyd;
  MSG_TRY(upload(ctx, dxd, x, (size_t)m->n_dofs));
  MSG_TRY(dxn.alloc(ctx, sizeof(double) * n3));
  MSG_TRY(dyn.alloc(ctx, sizeof(double) * n3));
  MSG_TRY(dyd.alloc(ctx, sizeof(double) * std::max(1, m->n_dofs)));
  MSG_CUDA(ctx, cudaMemsetAsync(dxn.ptr, 0, sizeof(double) * n3, ctx->stream));
  MSG_TRY(launch_dof_to_node(ctx, m, dxd.as<double>(), dxn.as<double>(), 1, 0, 0));
  MSG_TRY(launch_bsr_spmv(ctx, m, A->d_val.as<double>(), dxn.as<double>(), dyn.as<double>()));
  MSG_TRY(launch_node_to_dof(ctx, m, dyn.as<double>(), dyd.as<double>(), 1, 0, 0));
  MSG_CUDA(ctx, cudaMemcpyAsync(y, dyd.ptr, sizeof(double) * m->n_dofs, cudaMemcpyDeviceToHost, ctx->stream));
  MSG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return MSG_OK;
}

int MSG_MAT_DIAGONAL(MSG_MAT A, double* diag) {
  if (!A || !diag) return MSG_ERR_INVALID_ARGUMENT;
  Mesh* m = A->mesh;
  Context* ctx = m->ctx;
  CTX_GUARD(ctx);
  std::vector<double> dinv(3 * (size_t)m->n_nodes);
  MSG_CUDA(ctx, cudaMemcpyAsync(dinv.data(), A->d_dinv.ptr, sizeof(double) * dinv.size(), cudaMemcpyDeviceToHost,
                                ctx->stream));
  MSG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  for (int i = 0; i < m->n_nodes; ++i)
    for (int c = 0; c < 3; ++c) {
      const int d = m->dof[3 * i + c];
      if (d >= 0) diag[d] = 1.0 / dinv[3 * i + c];
    }
  return MSG_OK;
}

int MSG_MAT_DESTROY(MSG_MAT A) {
  if (!A) return MSG_ERR_INVALID_ARGUMENT;
  Mesh* m = A->mesh;
  Context* ctx = m->ctx;
  {
    std::lock_guard<std::recursive_mutex> lk(ctx->mu);
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    delete A;
  }
  release(m);
  return MSG_OK;
}

static int pcg_host(MSG_MAT A, const double* b, double* x, int max_it, double tol, int* iterations, double* rel_res,
                    bool mixed) {
  if (!A || !b || !x || max_it <= 0 || !(tol > 0)) return MSG_ERR_INVALID_ARGUMENT;
  Mesh* m = A->mesh;
  Context* ctx = m->ctx;
  CTX_GUARD(ctx);
  const size_t n3 = 3 * (size_t)m->n_nodes;
  // node-layout b / x and DOF staging kept with the matrix (no per-call allocation, graph reuse)
  if (!A->d_bn.ptr) {
    MSG_TRY(A->d_bd.alloc(ctx, sizeof(double) * std::max(1, m->n_dofs)));
    MSG_TRY(A->d_bn.alloc(ctx, sizeof(double) * n3));
    MSG_TRY(A->d_xn.alloc(ctx, sizeof(double) * n3));
    MSG_CUDA(ctx, cudaMemsetAsync(A->d_bn.ptr, 0, sizeof(double) * n3, ctx->stream));
  }
  MSG_CUDA(ctx, cudaMemcpyAsync(A->d_bd.ptr, b, sizeof(double) * m->n_dofs, cudaMemcpyHostToDevice, ctx->stream));
  MSG_TRY(launch_dof_to_node(ctx, m, A->d_bd.as<double>(), A->d_bn.as<double>(), 1, 0, 0));
  int its = 0, st = 0;
  double rr = 0;
  MSG_TRY(pcg_solve_device(ctx, A, A->d_bn.as<double>(), A->d_xn.as<double>(), max_it, tol, &its, &rr, &st, mixed));
  MSG_TRY(launch_node_to_dof(ctx, m, A->d_xn.as<double>(), A->d_bd.as<double>(), 1, 0, 0));
  MSG_CUDA(ctx, cudaMemcpyAsync(x, A->d_bd.ptr, sizeof(double) * m->n_dofs, cudaMemcpyDeviceToHost, ctx->stream));
  MSG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  if (iterations) *iterations = its;
  if (rel_res) *rel_res = rr;
  if (st != MSG_OK)
    return set_error(ctx, st, st == MSG_ERR_BREAKDOWN ? "PCG breakdown (p.q <= 0 or NaN)" : "PCG did not converge");
  return MSG_OK;
}

int MSG_PCG_SOLVE(MSG_MAT A, const double* b, double* x, int max_it, double tol, int* iterations, double* rel_res) {
  return pcg_host(A, b, x, max_it, tol, iterations, rel_res, false);
}

int MSG_PCG_SOLVE_MIXED(MSG_MAT A, const double* b, double* x, int max_it, double tol, int* iterations,
                        double* rel_res) {
  return pcg_host(A, b, x, max_it, tol, iterations, rel_res, true);
}

int MSG_PC_SIZE(int m, int p, int* size) {
  if (!size) return MSG_ERR_INVALID_ARGUMENT;
  const int P = pc_size(m, p);
  if (P < 0) return MSG_ERR_INVALID_ARGUMENT;
  *size = P;
  return MSG_OK;
}

int MSG_PC_BASIS(int m, int p, int* basis, int* norms) {
  std::vector<int> b, n;
  if (pc_basis(m, p, b, n) != MSG_OK) return MSG_ERR_INVALID_ARGUMENT;
  if (basis) std::memcpy(basis, b.data(), sizeof(int) * b.size());
  if (norms) std::memcpy(norms, n.data(), sizeof(int) * n.size());
  return MSG_OK;
}

int MSG_PC_GALERKIN_MATVEC(MSG_MESH mesh, double nu, const MSG_KL* kl, int m, int p, const double* u, double* y) {
  if (!mesh || !kl || !u || !y) return MSG_ERR_INVALID_ARGUMENT;
  Context* ctx = mesh->ctx;
  CTX_GUARD(ctx);
  if (!(nu > -1.0 && nu < 0.5)) return set_error(ctx, MSG_ERR_INVALID_ARGUMENT, "Poisson ratio out of (-1, 0.5)");
  return pc_matvec(ctx, mesh, nu, kl, m, p, u, y);
}

int MSG_SVS_CREATE(MSG_MESH mesh, int capacity, MSG_SVS* out) {
  if (!mesh || !out) return MSG_ERR_INVALID_ARGUMENT;
  Context* ctx = mesh->ctx;
  CTX_GUARD(ctx);
  SearchVectorStore* s = nullptr;
  MSG_TRY(svs_create(ctx, mesh, capacity, &s));
  *out = static_cast<MSG_SVS>(s);
  return MSG_OK;
}

int MSG_SVS_CLEAR(MSG_SVS store, int keep_from_top) {
  if (!store) return MSG_ERR_INVALID_ARGUMENT;
  Context* ctx = store->mesh->ctx;
  CTX_GUARD(ctx);
  store->count = keep_from_top < 1 ? 0 : std::min(store->count, keep_from_top);
  return MSG_OK;
}

int MSG_SVS_COUNT(MSG_SVS store, int* count) {
  if (!store || !count) return MSG_ERR_INVALID_ARGUMENT;
  *count = store->count;
  return MSG_OK;
}

int MSG_SVS_DESTROY(MSG_SVS store) {
  if (!store) return MSG_OK;
  Context* ctx = store->mesh->ctx;
  {
    CTX_GUARD(ctx);
    cudaStreamSynchronize(ctx->stream);
  }
  delete static_cast<SearchVectorStore*>(store);
  return MSG_OK;
}

int MSG_PCG_SOLVE_REORTH(MSG_MAT A, MSG_SVS store, const double* b, double* x, int start_from_store, int max_it,
                         double tol, int* iterations, double* rel_res) {
  if (!A || !store || !b || !x || max_it <= 0 || !(tol > 0)) return MSG_ERR_INVALID_ARGUMENT;
  Mesh* m = A->mesh;
  Context* ctx = m->ctx;
  CTX_GUARD(ctx);
  if (store->mesh != m) return set_error(ctx, MSG_ERR_INVALID_ARGUMENT, "search vector store belongs to another mesh");
  const size_t n3 = 3 * (size_t)m->n_nodes;
  if (!A->d_bn.ptr) {
    MSG_TRY(A->d_bd.alloc(ctx, sizeof(double) * std::max(1, m->n_dofs)));
    MSG_TRY(A->d_bn.alloc(ctx, sizeof(double) * n3));
    MSG_TRY(A->d_xn.alloc(ctx, sizeof(double) * n3));
    MSG_CUDA(ctx, cudaMemsetAsync(A->d_bn.ptr, 0, sizeof(double) * n3, ctx->stream));
  }
  MSG_CUDA(ctx, cudaMemcpyAsync(A->d_bd.ptr, b, sizeof(double) * m->n_dofs, cudaMemcpyHostToDevice, ctx->stream));
  MSG_TRY(launch_dof_to_node(ctx, m, A->d_bd.as<double>(), A->d_bn.as<double>(), 1, 0, 0));
  if (start_from_store < 0 || start_from_store > 2)
    return set_error(ctx, MSG_ERR_INVALID_ARGUMENT, "start_from_store must be 0, 1 or 2");
  const int st = pcg_reorth_solve(ctx, A, store, A->d_bn.as<double>(), A->d_xn.as<double>(), start_from_store,
                                  max_it, tol, iterations, rel_res);
  if (st != MSG_OK && st != MSG_ERR_NOT_CONVERGED) return st;
  MSG_TRY(launch_node_to_dof(ctx, m, A->d_xn.as<double>(), A->d_bd.as<double>(), 1, 0, 0));
  MSG_CUDA(ctx, cudaMemcpyAsync(x, A->d_bd.ptr, sizeof(double) * m->n_dofs, cudaMemcpyDeviceToHost, ctx->stream));
  MSG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return st;
}

int MSG_KL_TABLE(const double* L, double l, int n_terms, int n1d, double* w3, double* amp3, int* idx3, double* eig) {
  if (!L || !(l > 0) || n_terms <= 0 || n1d <= 0 || !w3 || !amp3 || !idx3 || !eig) return MSG_ERR_INVALID_ARGUMENT;
  if ((int64_t)n1d * n1d * n1d < n_terms) return MSG_ERR_INVALID_ARGUMENT;
  const double pi = 3.14159265358979323846;
  const double c = 1.0 / l;
  std::vector<double> w[3], a[3], lam[3];
  for (int ax = 0; ax < 3; ++ax) {
    if (!(L[ax] > 0)) return MSG_ERR_INVALID_ARGUMENT;
    const double A = 0.5 * L[ax];
    for (int k = 1; k <= n1d; ++k) {
      const bool is_sin = (k % 2 == 0);
      const int i = k / 2;
      const double lo = is_sin ? (i - 0.5) * pi / A : i * pi / A;
      const double hi = is_sin ? i * pi / A : (i + 0.5) * pi / A;
      const double ww = kl_root(A, c, is_sin, lo, hi);
      const double s = std::sin(2.0 * ww * A) / (2.0 * ww);
      w[ax].push_back(ww);
      lam[ax].push_back(2.0 * c / (ww * ww + c * c));
      a[ax].push_back(1.0 / std::sqrt(is_sin ? A - s : A + s));
    }
  }
  struct Term { int64_t key; int i, j, k; double e; };
  std::vector<Term> t;
  t.reserve((size_t)n1d * n1d * n1d);
  const double emax = lam[0][0] * lam[1][0] * lam[2][0];
  for (int i = 0; i < n1d; ++i)
    for (int j = 0; j < n1d; ++j)
      for (int k = 0; k < n1d; ++k) {
        const double e = (lam[0][i] * lam[1][j]) * lam[2][k];
        t.push_back({(int64_t)std::llround(e / emax * 1099511627776.0), i, j, k, e});  // 2^-40 quantised key
      }
  std::sort(t.begin(), t.end(), [](const Term& x, const Term& y) {
    if (x.key != y.key) return x.key > y.key;
    if (x.i != y.i) return x.i < y.i;
    if (x.j != y.j) return x.j < y.j;
    return x.k < y.k;
  });
  for (int q = 0; q < n_terms; ++q) {
    const int id[3] = {t[q].i, t[q].j, t[q].k};
    for (int ax = 0; ax < 3; ++ax) {
      w3[3 * q + ax] = w[ax][id[ax]];
      amp3[3 * q + ax] = a[ax][id[ax]];
      idx3[3 * q + ax] = id[ax] + 1;
    }
    eig[q] = t[q].e;
  }
  return MSG_OK;
}

int MSG_KL_FIELD(MSG_MESH m, const MSG_KL* kl, int R, const double* xi, double* E) {
  if (!m || !kl || R <= 0 || !xi || !E) return MSG_ERR_INVALID_ARGUMENT;
  Context* ctx = m->ctx;
  CTX_GUARD(ctx);
  KLDevice kd;
  MSG_TRY(kl_prepare(ctx, m, kl, &kd));
  const int Rp = (R + 31) / 32 * 32;
  DevMem dxi, dE;
  MSG_TRY(upload(ctx, dxi, xi, (size_t)R * kl->n_terms));
  MSG_TRY(dE.alloc(ctx, sizeof(double) * (size_t)R * m->n_elems));
  MSG_TRY(launch_kl_field(ctx, m, &kd, R, Rp, dxi.as<double>(), nullptr, nullptr, dE.as<double>()));
  MSG_CUDA(ctx, cudaMemcpyAsync(E, dE.ptr, sizeof(double) * (size_t)R * m->n_elems, cudaMemcpyDeviceToHost, ctx->stream));
  MSG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return MSG_OK;
}

int MSG_MC_SOLVE_BATCH_DEVICE(MSG_MESH m, double nu, const MSG_KL* kl, int R, const double* xi_dev, const double* b_dev,
                              int mode, int max_it, double tol, int tip_dof, double* X_dev, double* tip,
                              int* iterations, double* rel_res) {
  if (!m) return MSG_ERR_INVALID_ARGUMENT;
  Context* ctx = m->ctx;
  CTX_GUARD(ctx);
  return mc_batch(ctx, m, nu, kl, R, xi_dev, b_dev, mode, max_it, tol, tip_dof, X_dev, tip, iterations, rel_res);
}

int MSG_MC_SOLVE_BATCH(MSG_MESH m, double nu, const MSG_KL* kl, int R, const double* xi, const double* b, int mode,
                       int max_it, double tol, int tip_dof, double* X, double* tip, int* iterations, double* rel_res) {
  if (!m || !kl || !xi || !b || R <= 0) return MSG_ERR_INVALID_ARGUMENT;
  Context* ctx = m->ctx;
  CTX_GUARD(ctx);
  MSG_TRY(pipe_flush(ctx));  // a pipelined call's copy may still read slot 14
  // staging buffers kept in the context (slots 12-14) across calls
  void *dxi = nullptr, *db = nullptr, *dX = nullptr;
  MSG_TRY(workspace(ctx, 12, sizeof(double) * (size_t)R * kl->n_terms, &dxi));
  MSG_TRY(workspace(ctx, 13, sizeof(double) * (size_t)std::max(1, m->n_dofs), &db));
  if (X) MSG_TRY(workspace(ctx, 14, sizeof(double) * (size_t)R * m->n_dofs, &dX));
  MSG_CUDA(ctx, cudaMemcpyAsync(dxi, xi, sizeof(double) * (size_t)R * kl->n_terms, cudaMemcpyHostToDevice, ctx->stream));
  MSG_CUDA(ctx, cudaMemcpyAsync(db, b, sizeof(double) * (size_t)m->n_dofs, cudaMemcpyHostToDevice, ctx->stream));
  int st = mc_batch(ctx, m, nu, kl, R, static_cast<double*>(dxi), static_cast<double*>(db), mode, max_it, tol, tip_dof,
                    X ? static_cast<double*>(dX) : nullptr, tip, iterations, rel_res);
  // per-realization outcomes (not converged, breakdown): the other realizations' results are valid
  if (X && (st == MSG_OK || st == MSG_ERR_NOT_CONVERGED || st == MSG_ERR_BREAKDOWN)) {
    MSG_CUDA(ctx, cudaMemcpyAsync(X, dX, sizeof(double) * (size_t)R * m->n_dofs, cudaMemcpyDeviceToHost, ctx->stream));
    MSG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  }
  return st;
}

int MSG_MC_SOLVE_BATCH_PIPELINED(MSG_MESH m, double nu, const MSG_KL* kl, int R, const double* xi, const double* b,
                                 int mode, int max_it, double tol, int tip_dof, double* X, double* tip,
                                 int* iterations, double* rel_res) {
  if (!m || !kl || !xi || !b || R <= 0) return MSG_ERR_INVALID_ARGUMENT;
  Context* ctx = m->ctx;
  CTX_GUARD(ctx);
  MSG_TRY(context_resources(ctx));
  if (!ctx->copy_stream) MSG_CUDA(ctx, cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking));
  for (auto& e : ctx->pipe_ev)
    if (!e) MSG_CUDA(ctx, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  if (!ctx->pipe_ready) MSG_CUDA(ctx, cudaEventCreateWithFlags(&ctx->pipe_ready, cudaEventDisableTiming));
  const int buf = ctx->pipe_next, other = buf ^ 1;
  void *dxi = nullptr, *db = nullptr, *dX = nullptr;
  MSG_TRY(workspace(ctx, 12, sizeof(double) * (size_t)R * kl->n_terms, &dxi));
  MSG_TRY(workspace(ctx, 13, sizeof(double) * (size_t)std::max(1, m->n_dofs), &db));
  if (X) {
    // output buffer `buf` (slot 14 or 36): its copy from two calls ago must have
    // left for the host before this batch writes it (a device-side wait)
    if (ctx->pipe_pending[buf]) MSG_CUDA(ctx, cudaStreamWaitEvent(ctx->stream, ctx->pipe_ev[buf], 0));
    MSG_TRY(workspace(ctx, buf ? 36 : 14, sizeof(double) * (size_t)R * std::max(1, m->n_dofs), &dX));
  }
  MSG_CUDA(ctx, cudaMemcpyAsync(dxi, xi, sizeof(double) * (size_t)R * kl->n_terms, cudaMemcpyHostToDevice, ctx->stream));
  MSG_CUDA(ctx, cudaMemcpyAsync(db, b, sizeof(double) * (size_t)m->n_dofs, cudaMemcpyHostToDevice, ctx->stream));
  int st = mc_batch(ctx, m, nu, kl, R, static_cast<double*>(dxi), static_cast<double*>(db), mode, max_it, tol,
                    tip_dof, X ? static_cast<double*>(dX) : nullptr, tip, iterations, rel_res);
  if (X && (st == MSG_OK || st == MSG_ERR_NOT_CONVERGED || st == MSG_ERR_BREAKDOWN)) {
    // the copy to the host follows the batch on the copy stream and is left in flight
    MSG_CUDA(ctx, cudaEventRecord(ctx->pipe_ready, ctx->stream));
    MSG_CUDA(ctx, cudaStreamWaitEvent(ctx->copy_stream, ctx->pipe_ready, 0));
    MSG_CUDA(ctx, cudaMemcpyAsync(X, dX, sizeof(double) * (size_t)R * m->n_dofs, cudaMemcpyDeviceToHost,
                                  ctx->copy_stream));
    MSG_CUDA(ctx, cudaEventRecord(ctx->pipe_ev[buf], ctx->copy_stream));
    ctx->pipe_pending[buf] = true;
  }
  // the previous call's copy (overlapped with this batch) is complete on return
  if (ctx->pipe_pending[other]) {
    ctx->pipe_pending[other] = false;
    MSG_CUDA(ctx, cudaEventSynchronize(ctx->pipe_ev[other]));
  }
  ctx->pipe_next = other;
  return st;
}

int MSG_MC_FLUSH(MSG_CTX ctx) {
  CTX_GUARD(ctx);
  return pipe_flush(ctx);
}

int MSG_MC_SOLVE_RAGGED(MSG_CTX ctx, int n_systems, const MSG_RAGGED_SYSTEM* systems, int max_it, double tol) {
  CTX_GUARD(ctx);
  if (n_systems <= 0 || !systems || max_it <= 0 || !(tol > 0))
    return set_error(ctx, MSG_ERR_INVALID_ARGUMENT, "ragged batch: invalid arguments");
  MSG_TRY(context_resources(ctx));
  MSG_TRY(pipe_flush(ctx));
  cudaEvent_t e0 = ctx->ev[12], e1 = ctx->ev[13];
  cudaEventRecord(e0, ctx->stream);
  for (int i = 0; i < n_systems; ++i) {
    const MSG_RAGGED_SYSTEM& y = systems[i];
    Mesh* m = y.mesh;
    if (!m || m->ctx != ctx || !y.kl || !y.xi || !y.b || y.R <= 0 || y.kl->n_terms <= 0)
      return set_error(ctx, MSG_ERR_INVALID_ARGUMENT, "ragged batch: invalid system %d", i);
    if (y.tip && y.tip_dof >= m->n_dofs) return set_error(ctx, MSG_ERR_INVALID_ARGUMENT, "tip_dof out of range");
  }
  // every system's xi, b and X staged in one workspace slot (kept across calls)
  auto up = [](size_t b) { return (b + 255) / 256 * 256; };
  std::vector<size_t> off(3 * (size_t)n_systems);
  size_t total = 0;
  for (int i = 0; i < n_systems; ++i) {
    const MSG_RAGGED_SYSTEM& y = systems[i];
    const size_t nd = (size_t)std::max(1, y.mesh->n_dofs);
    off[3 * i] = total;
    total += up(sizeof(double) * (size_t)y.R * y.kl->n_terms);
    off[3 * i + 1] = total;
    total += up(sizeof(double) * nd);
    off[3 * i + 2] = total;
    if (y.X) total += up(sizeof(double) * (size_t)y.R * nd);
  }
  void* stage = nullptr;
  MSG_TRY(workspace(ctx, 37, total, &stage));
  unsigned char* base = static_cast<unsigned char*>(stage);
  std::vector<RgInput> in;  // the systems of the shared element-by-element batch
  std::vector<int> lattice;  // cube lattices solved by the lattice loop
  for (int i = 0; i < n_systems; ++i) {
    const MSG_RAGGED_SYSTEM& y = systems[i];
    Mesh* m = y.mesh;
    double* dxi = reinterpret_cast<double*>(base + off[3 * i]);
    double* db = reinterpret_cast<double*>(base + off[3 * i + 1]);
    MSG_CUDA(ctx, cudaMemcpyAsync(dxi, y.xi, sizeof(double) * (size_t)y.R * y.kl->n_terms, cudaMemcpyHostToDevice,
                                  ctx->stream));
    MSG_CUDA(ctx, cudaMemcpyAsync(db, y.b, sizeof(double) * (size_t)m->n_dofs, cudaMemcpyHostToDevice, ctx->stream));
    if (ctx->ragged_lattice_loop && m->structured) {
      lattice.push_back(i);
      continue;
    }
    RgInput I;
    I.m = m;
    I.nu = y.nu;
    I.kl = y.kl;
    I.R = y.R;
    I.d_xi = dxi;
    I.d_b = db;
    I.d_X = y.X ? reinterpret_cast<double*>(base + off[3 * i + 2]) : nullptr;
    I.h_tip = y.tip;
    I.tip_dof = y.tip ? y.tip_dof : -1;
    I.h_its = y.iterations;
    I.h_res = y.rel_res;
    in.push_back(I);
  }
  // per-realization outcomes (not converged, breakdown) leave every other output complete
  int worst = MSG_OK;
  auto outcome = [&](int st) {
    if (st != MSG_OK && st != MSG_ERR_NOT_CONVERGED && st != MSG_ERR_BREAKDOWN) return false;
    if (worst == MSG_OK) worst = st;
    return true;
  };
  if (ctx->ragged_side_by_side && !lattice.empty() && (lattice.size() > 1 || !in.empty())) {
    // the cube lattices' loops stepped side by side, each on its own stream, on
    // a second host thread while this one runs the element-by-element batch
    std::vector<LatticeJob> jobs;
    for (int i : lattice) {
      const MSG_RAGGED_SYSTEM& y = systems[i];
      LatticeJob J;
      J.m = y.mesh;
      J.nu = y.nu;
      J.kl = y.kl;
      J.R = y.R;
      J.d_xi = reinterpret_cast<double*>(base + off[3 * i]);
      J.d_b = reinterpret_cast<double*>(base + off[3 * i + 1]);
      J.d_X = y.X ? reinterpret_cast<double*>(base + off[3 * i + 2]) : nullptr;
      J.h_tip = y.tip;
      J.tip_dof = y.tip ? y.tip_dof : -1;
      J.h_its = y.iterations;
      J.h_res = y.rel_res;
      jobs.push_back(J);
    }
    int ebe_status = MSG_OK;
    std::function<int()> ebe;
    if (!in.empty()) ebe = [&] { return ebe_status = ebe_solve(ctx, in, max_it, tol); };
    const int st = block_mixed_solve_many(ctx, jobs, max_it, tol, ebe);
    // a status of the element-by-element batch is its outcome, any other a failure
    if (st != MSG_OK && st != ebe_status) return st;
    for (const LatticeJob& J : jobs)
      if (!outcome(J.status)) return J.status;
    if (!in.empty() && !outcome(ebe_status)) return ebe_status;
    in.clear();  // solved
  } else {
    for (int i : lattice) {
      const MSG_RAGGED_SYSTEM& y = systems[i];
      const int st = mc_batch(ctx, y.mesh, y.nu, y.kl, y.R, reinterpret_cast<double*>(base + off[3 * i]),
                              reinterpret_cast<double*>(base + off[3 * i + 1]), MSG_MODE_MIXED_BATCHED, max_it, tol,
                              y.tip ? y.tip_dof : -1,
                              y.X ? reinterpret_cast<double*>(base + off[3 * i + 2]) : nullptr, y.tip, y.iterations,
                              y.rel_res);
      if (!outcome(st)) return st;
    }
  }
  if (!in.empty()) {
    const int st = ebe_solve(ctx, in, max_it, tol);
    if (!outcome(st)) return st;
  }
  for (int i = 0; i < n_systems; ++i)
    if (systems[i].X)
      MSG_CUDA(ctx, cudaMemcpyAsync(systems[i].X, base + off[3 * i + 2],
                                    sizeof(double) * (size_t)systems[i].R * systems[i].mesh->n_dofs,
                                    cudaMemcpyDeviceToHost, ctx->stream));
  cudaEventRecord(e1, ctx->stream);
  cudaEventSynchronize(e1);
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  ctx->t_phase[4] = ms;
  return worst;
}

int MSG_NEWMARK_BATCH(MSG_MESH m, double nu, const MSG_KL* kl, int R, const double* xi, const MSG_NEWMARK* nm,
                      const double* f_static, int max_it, double tol, int tip_dof, double* tip_hist, double* U,
                      int* iterations) {
  if (!m || !kl || !xi || !nm || R <= 0 || max_it <= 0 || !(tol > 0)) return MSG_ERR_INVALID_ARGUMENT;
  Context* ctx = m->ctx;
  CTX_GUARD(ctx);
  if (!m->structured) return set_error(ctx, MSG_ERR_NOT_STRUCTURED, "Newmark batch needs a structured cube lattice");
  if (tip_dof >= m->n_dofs) return set_error(ctx, MSG_ERR_INVALID_ARGUMENT, "tip_dof out of range");
  // realizations padded to 64: the packed level operator works on pairs of 32-wide groups
  const int Rp = (R + 63) / 64 * 64;
  MSG_TRY(context_resources(ctx));
  cudaEvent_t e0 = ctx->ev[8], e1 = ctx->ev[9];
  cudaEventRecord(e0, ctx->stream);
  void *dxi = nullptr, *df = nullptr, *dU = nullptr;
  MSG_TRY(workspace(ctx, 12, sizeof(double) * (size_t)R * kl->n_terms, &dxi));
  MSG_CUDA(ctx, cudaMemcpyAsync(dxi, xi, sizeof(double) * (size_t)R * kl->n_terms, cudaMemcpyHostToDevice, ctx->stream));
  if (f_static) {
    MSG_TRY(workspace(ctx, 13, sizeof(double) * (size_t)std::max(1, m->n_dofs), &df));
    MSG_CUDA(ctx, cudaMemcpyAsync(df, f_static, sizeof(double) * (size_t)m->n_dofs, cudaMemcpyHostToDevice,
                                  ctx->stream));
  }
  if (U) MSG_TRY(workspace(ctx, 14, sizeof(double) * (size_t)R * m->n_dofs, &dU));
  KLDevice kd;
  MSG_TRY(kl_prepare(ctx, m, kl, &kd));
  NewmarkParams p;
  p.rho = nm->rho;
  p.ray_alpha = nm->rayleigh_alpha;
  p.ray_beta = nm->rayleigh_beta;
  p.alpha = nm->alpha;
  p.delta = nm->delta;
  p.dt = nm->dt;
  p.n_steps = nm->n_steps;
  p.acc_amp = nm->acc_amp;
  p.acc_period = nm->acc_period;
  p.acc_dir = nm->acc_dof;
  int st = block_newmark(ctx, m, nu, &kd, static_cast<double*>(dxi), R, Rp, p, static_cast<double*>(df), max_it, tol,
                         tip_dof, tip_hist, static_cast<double*>(dU), iterations);
  if (U && st == MSG_OK) {
    MSG_CUDA(ctx, cudaMemcpyAsync(U, dU, sizeof(double) * (size_t)R * m->n_dofs, cudaMemcpyDeviceToHost, ctx->stream));
    MSG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  }
  cudaEventRecord(e1, ctx->stream);
  cudaEventSynchronize(e1);
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  ctx->t_phase[4] = ms;
  return st;
}

}  // extern "C"
