// Slab parts of a structured-grid tissue: the row distribution of the
// reference's parallel solve (PETSc MPIAIJ rows split with PETSC_DECIDE,
// fem.cpp:667-670; MatMult and KSPSolve exchange ghost values and reduce
// the CG dot products across ranks, fem.cpp:705-718) restated as device
// kernels for one part, with the exchange left to the caller.
//
// A part owns a contiguous range of planes of the grid (the last axis: y in
// 2D, z in 3D), planes divided as PETSC_DECIDE divides rows. Its rows of A
// and B come from the grid assembly kernel run on that row range, so they
// are bit-identical to the same rows of the whole operator; columns index
// the part's extended vector [lower halo plane | owned rows | upper halo
// plane]. The solve is the Jacobi-PCG of the whole-operator path (zero
// start, b = B V / dt, the same stopping rule) split into three kernels per
// iteration (direction, product, update). Between them the caller moves
// the boundary planes of p to the neighbouring parts and gathers every
// part's partial sums ([n_parts][2] doubles, in part order); every kernel
// adds the parts' partials in part order, so all parts take the same
// decisions and the result does not depend on how parts map to ranks. Each
// kernel reduces its own rows in a fixed order (a fixed grid and the last
// block summing the block partials in block order): a part's partials are
// the same from run to run.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <vector>

#include "../../include/cep_b200.h"
#include "internal.h"

extern "C" int cep_internal_fem_assemble_grid_rows(int dim, int nx, int ny, int nz, double h, double dt,
                                                   const double *d_D, int n_d, int64_t e_off, int64_t row0,
                                                   int64_t n_rows, int64_t col_off, const int *d_rp, int *d_col,
                                                   double *d_a, double *d_b, int width, int64_t ld, int *d_ecol,
                                                   double *d_ea, double *d_eb, double *d_dinv, void *stream);

namespace {

int fail_msg(int code, const char *fmt, ...) {
  char buf[400];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  return cep_internal_set_fail(code, buf);
}

#define SLAB_CUDA(call)                                                                         \
  do {                                                                                          \
    cudaError_t e_ = (call);                                                                    \
    if (e_ != cudaSuccess) return fail_msg(CEP_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
  } while (0)

constexpr int kBlock = 256;
constexpr int kMaxBlocks = 296;  // two per SM: the fixed grid of every reduction

// CG scalars of a part, double-buffered by iteration parity: the direction
// kernel of host iteration j reads copy j & 1 and writes copy (j + 1) & 1.
struct State {
  double rz, n0, res;
  int used, done, conv, pad;
};

}  // namespace

struct cep_part {
  int dim = 0, nx = 0, ny = 0, nz = 0, part = 0, n_parts = 0;
  int64_t plane = 0, row0 = 0, n_own = 0, lo = 0, hi = 0, ld = 0;
  int width = 0, nb = 1;
  double dt = 0.0, rtol = 1e-5;
  int max_iter = 10000, precond_norm = 1;
  cudaStream_t stream = nullptr;
  int *rp = nullptr, *col = nullptr, *ecol = nullptr;
  double *a = nullptr, *b = nullptr, *ea = nullptr, *eb = nullptr, *dinv = nullptr;
  double *x = nullptr, *r = nullptr, *z = nullptr, *q = nullptr, *p = nullptr;
  double *scratch = nullptr;    // [kMaxBlocks][2] block partials
  unsigned *counter = nullptr;  // blocks finished (the last one reduces)
  State *st = nullptr;          // [2]
  int64_t nnz = 0;
  // tissue binding
  cep_batch_t cells = nullptr;
  unsigned char *mask = nullptr;
  double bcl = 1000.0, t_crt = 0.0, dur = 0.0;
  int n_pace = 1;
  double *tact = nullptr, act_thr = 0.0;
  std::vector<void *> allocs;
};

namespace cep {
namespace slab {

__device__ __forceinline__ void block_sum2(double &a, double &b) {
  __shared__ double sa[kBlock], sb[kBlock];
  sa[threadIdx.x] = a;
  sb[threadIdx.x] = b;
  __syncthreads();
  for (int w = kBlock / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) {
      sa[threadIdx.x] += sa[threadIdx.x + w];
      sb[threadIdx.x] += sb[threadIdx.x + w];
    }
    __syncthreads();
  }
  a = sa[0];
  b = sb[0];
  __syncthreads();
}

// The block partials of a kernel: the last block to finish adds them in
// block order and writes the part's two partial sums.
__device__ void finish_partials(double s0, double s1, double *scratch, unsigned *counter, double *out) {
  __shared__ bool last;
  block_sum2(s0, s1);
  if (threadIdx.x == 0) {
    scratch[2 * blockIdx.x] = s0;
    scratch[2 * blockIdx.x + 1] = s1;
    __threadfence();
    last = atomicAdd(counter, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  double t0 = 0.0, t1 = 0.0;
  for (int k = threadIdx.x; k < (int)gridDim.x; k += kBlock) {
    t0 += ((volatile double *)scratch)[2 * k];
    t1 += ((volatile double *)scratch)[2 * k + 1];
  }
  block_sum2(t0, t1);
  if (threadIdx.x == 0) {
    out[0] = t0;
    out[1] = t1;
    *counter = 0;
  }
}

// the parts' partials added in part order
__device__ __forceinline__ void total2(const double *all, int n_parts, double &s0, double &s1) {
  s0 = 0.0;
  s1 = 0.0;
  for (int k = 0; k < n_parts; ++k) {
    s0 += all[2 * k];
    s1 += all[2 * k + 1];
  }
}

struct View {
  const int *ecol;
  const double *ea, *eb, *dinv;
  int64_t n_own, lo, ld;
  int width;
};

// sum over the row's slots of m[s][i] * v[col], v given as the lower halo
// plane, the owned rows and the upper halo plane
__device__ __forceinline__ double row_apply(const View &w, const double *m, int64_t i, const double *vlo,
                                            const double *vown, const double *vhi) {
  double acc = 0.0;
  for (int s = 0; s < w.width; ++s) {
    const int64_t c = w.ecol[(int64_t)s * w.ld + i];
    const double v = c < w.lo ? vlo[c] : (c >= w.lo + w.n_own ? vhi[c - w.lo - w.n_own] : vown[c - w.lo]);
    acc = fma(m[(int64_t)s * w.ld + i], v, acc);
  }
  return acc;
}

// b = B V / dt, r = b, z = D^-1 b, x = 0, p = 0; partials (r.z, |z|^2 or |r|^2)
__global__ void __launch_bounds__(kBlock) begin_kernel(View w, double dt, int precond_norm, const double *v,
                                                       const double *vlo, const double *vhi, double *x, double *r,
                                                       double *z, double *p, State *st, double *scratch,
                                                       unsigned *counter, double *out) {
  double s0 = 0.0, s1 = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * kBlock + threadIdx.x; i < w.n_own; i += (int64_t)gridDim.x * kBlock) {
    const double bi = row_apply(w, w.eb, i, vlo, v, vhi) / dt;
    const double zi = w.dinv[i] * bi;
    r[i] = bi;
    z[i] = zi;
    x[i] = 0.0;
    p[i] = 0.0;
    s0 = fma(bi, zi, s0);
    s1 = precond_norm ? fma(zi, zi, s1) : fma(bi, bi, s1);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) st[0] = State{0.0, 0.0, 0.0, 0, 0, 0, 0};
  finish_partials(s0, s1, scratch, counter, out);
}

// Iteration j's scalars from the parts' partials, then p = z + beta p and
// the boundary planes of p into the send buffers.
__global__ void __launch_bounds__(kBlock) direction_kernel(int64_t n_own, int64_t plane, int j, const double *all,
                                                           int n_parts, double rtol, int max_iter, const double *z,
                                                           double *p, State *st, double *send_lo, double *send_hi) {
  const State s = st[j & 1];
  State t = s;
  double beta = 0.0;
  if (!s.done) {
    double a0, a1;
    total2(all, n_parts, a0, a1);
    if (j == 0) {  // the partials of the start: r.z and the initial norm
      t.rz = a0;
      t.n0 = sqrt(a1);
      t.res = t.n0 > 0.0 ? 1.0 : 0.0;
      if (t.n0 == 0.0) t.done = t.conv = 1;
    } else {  // the partials of update j - 1: r.z and the residual norm
      const double nr = sqrt(a1);
      t.res = nr / s.n0;
      t.used = j;
      if (nr <= rtol * s.n0) {
        t.done = t.conv = 1;
      } else if (j >= max_iter) {
        t.done = 1;
      }
      beta = a0 / s.rz;
      t.rz = a0;
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) st[(j + 1) & 1] = t;
  if (t.done) return;
  for (int64_t i = (int64_t)blockIdx.x * kBlock + threadIdx.x; i < n_own; i += (int64_t)gridDim.x * kBlock) {
    const double pi = fma(beta, p[i], z[i]);
    p[i] = pi;
    if (send_lo && i < plane) send_lo[i] = pi;
    if (send_hi && i >= n_own - plane) send_hi[i - (n_own - plane)] = pi;
  }
}

// q = A p over the extended vector; partial p.q
__global__ void __launch_bounds__(kBlock) product_kernel(View w, int j, const double *p, const double *plo,
                                                         const double *phi, double *q, const State *st,
                                                         double *scratch, unsigned *counter, double *out) {
  if (st[(j + 1) & 1].done) return;
  double s0 = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * kBlock + threadIdx.x; i < w.n_own; i += (int64_t)gridDim.x * kBlock) {
    const double qi = row_apply(w, w.ea, i, plo, p, phi);
    q[i] = qi;
    s0 = fma(p[i], qi, s0);
  }
  finish_partials(s0, 0.0, scratch, counter, out);
}

// alpha = r.z / p.q (the parts' sums); x += alpha p, r -= alpha q,
// z = D^-1 r; partials (r.z, |z|^2 or |r|^2)
__global__ void __launch_bounds__(kBlock) update_kernel(View w, int j, const double *all, int n_parts,
                                                        int precond_norm, const double *p, const double *q, double *x,
                                                        double *r, double *z, const State *st, double *scratch,
                                                        unsigned *counter, double *out) {
  const State s = st[(j + 1) & 1];
  if (s.done) return;
  double pq, unused;
  total2(all, n_parts, pq, unused);
  const double alpha = s.rz / pq;
  double s0 = 0.0, s1 = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * kBlock + threadIdx.x; i < w.n_own; i += (int64_t)gridDim.x * kBlock) {
    x[i] = fma(alpha, p[i], x[i]);
    const double ri = fma(-alpha, q[i], r[i]);
    const double zi = w.dinv[i] * ri;
    r[i] = ri;
    z[i] = zi;
    s0 = fma(ri, zi, s0);
    s1 = precond_norm ? fma(zi, zi, s1) : fma(ri, ri, s1);
  }
  finish_partials(s0, s1, scratch, counter, out);
}

__global__ void end_kernel(int64_t n_own, const double *x, double *v, double *tact, double t_new, double thr) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_own) return;
  const double vi = x[i];
  v[i] = vi;
  if (tact && tact[i] < 0.0 && vi >= thr) tact[i] = t_new;
}

__global__ void fill_kernel(int64_t n, double *y, double value) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) y[i] = value;
}

}  // namespace slab
}  // namespace cep

namespace {

template <class T>
int part_alloc(cep_part *p, T **ptr, size_t count) {
  void *q = nullptr;
  if (cudaMalloc(&q, count * sizeof(T) + 64) != cudaSuccess) {
    cudaGetLastError();
    return fail_msg(CEP_ERR_OOM, "slab part: cudaMalloc of %zu bytes", count * sizeof(T));
  }
  p->allocs.push_back(q);
  *ptr = static_cast<T *>(q);
  return CEP_OK;
}

void part_free(cep_part *p) {
  if (p->stream) cudaStreamSynchronize(p->stream);
  for (void *q : p->allocs) cudaFree(q);
  delete p;
}

cep::slab::View view_of(const cep_part *p) {
  return cep::slab::View{p->ecol, p->ea, p->eb, p->dinv, p->n_own, p->lo, p->ld, p->width};
}

unsigned grid_of(int64_t n) { return (unsigned)std::max<int64_t>(1, std::min<int64_t>(kMaxBlocks, (n + kBlock - 1) / kBlock)); }

}  // namespace

extern "C" {

int cep_part_split(int n_planes, int n_parts, int part, int *first_plane, int *planes) {
  if (n_planes < 1 || n_parts < 1 || n_parts > n_planes || part < 0 || part >= n_parts)
    return fail_msg(CEP_ERR_ARG, "cannot split %d planes into %d parts (part %d)", n_planes, n_parts, part);
  const int base = n_planes / n_parts, rem = n_planes % n_parts;
  if (first_plane) *first_plane = part * base + std::min(part, rem);
  if (planes) *planes = base + (part < rem ? 1 : 0);
  return CEP_OK;
}

int cep_part_create_grid(int dim, int nx, int ny, int nz, double h, double dt, const double *D, int n_d, int part,
                         int n_parts, void *stream, cep_part_t *out) {
  if (!out || !D) return fail_msg(CEP_ERR_ARG, "null argument");
  *out = nullptr;
  if (dim != 2 && dim != 3) return fail_msg(CEP_ERR_ARG, "dim must be 2 or 3 (got %d)", dim);
  if (dim == 2) nz = 1;
  if (nx < 2 || ny < 2 || (dim == 3 && nz < 2)) return fail_msg(CEP_ERR_ARG, "grid needs >= 2 nodes per axis");
  if (!(h > 0) || !(dt > 0)) return fail_msg(CEP_ERR_ARG, "h and dt must be positive");
  const int full = dim == 2 ? 3 : 6;
  if (n_d != 1 && n_d != full) return fail_msg(CEP_ERR_ARG, "n_d must be 1 or %d for dim %d", full, dim);
  const int64_t n = (int64_t)nx * ny * nz;
  if (n > 0x7fffffffLL / 27) return fail_msg(CEP_ERR_ARG, "grid too large for 32-bit column indices");
  const int n_planes = dim == 2 ? ny : nz;
  int p0 = 0, np = 0;
  if (int rc = cep_part_split(n_planes, n_parts, part, &p0, &np)) return rc;
  cep_part *p = new cep_part;
  p->dim = dim; p->nx = nx; p->ny = ny; p->nz = nz; p->part = part; p->n_parts = n_parts;
  p->plane = dim == 2 ? (int64_t)nx : (int64_t)nx * ny;
  p->row0 = (int64_t)p0 * p->plane;
  p->n_own = (int64_t)np * p->plane;
  p->lo = part > 0 ? p->plane : 0;
  p->hi = part < n_parts - 1 ? p->plane : 0;
  p->ld = (p->n_own + 31) / 32 * 32;
  p->width = dim == 2 ? 9 : 27;
  p->dt = dt;
  p->stream = (cudaStream_t)stream;
  p->nb = (int)grid_of(p->n_own);
  // row pointers of the owned rows (neighbours per axis: 1 + (i > 0) + (i < m-1))
  std::vector<int> rp((size_t)p->n_own + 1);
  int64_t q = 0;
  auto cnt = [](int i, int m) { return 1 + (i > 0) + (i < m - 1); };
  for (int64_t li = 0; li < p->n_own; ++li) {
    const int64_t i = p->row0 + li;
    const int ix = (int)(i % nx), iy = (int)((i / nx) % ny), iz = (int)(i / ((int64_t)nx * ny));
    rp[(size_t)li] = (int)q;
    q += (int64_t)cnt(ix, nx) * cnt(iy, ny) * (dim == 3 ? cnt(iz, nz) : 1);
  }
  rp[(size_t)p->n_own] = (int)q;
  p->nnz = q;
  // elements touching the owned planes: element planes p0-1 .. p0+np-1
  const int64_t eplane = dim == 2 ? (int64_t)(nx - 1) : (int64_t)(nx - 1) * (ny - 1);
  const int e_first = std::max(p0 - 1, 0), e_last = std::min(p0 + np, n_planes - 1);  // exclusive
  const int64_t e_off = (int64_t)e_first * eplane, n_e = (int64_t)(e_last - e_first) * eplane;
  for (int64_t e = e_off * n_d; e < (e_off + n_e) * n_d; ++e)
    if (!std::isfinite(D[e])) {
      delete p;
      return fail_msg(CEP_ERR_ARG, "D[%lld] is not finite", (long long)e);
    }
  int rc;
  int *d_rp = nullptr;
  double *d_D = nullptr;
  const size_t w = (size_t)p->width * p->ld;
  if ((rc = part_alloc(p, &d_rp, rp.size())) || (rc = part_alloc(p, &p->col, (size_t)q)) ||
      (rc = part_alloc(p, &p->a, (size_t)q)) || (rc = part_alloc(p, &p->b, (size_t)q)) ||
      (rc = part_alloc(p, &p->ecol, w)) || (rc = part_alloc(p, &p->ea, w)) || (rc = part_alloc(p, &p->eb, w)) ||
      (rc = part_alloc(p, &p->dinv, (size_t)p->ld)) || (rc = part_alloc(p, &d_D, (size_t)std::max<int64_t>(1, n_e * n_d))) ||
      (rc = part_alloc(p, &p->x, (size_t)p->ld)) || (rc = part_alloc(p, &p->r, (size_t)p->ld)) ||
      (rc = part_alloc(p, &p->z, (size_t)p->ld)) || (rc = part_alloc(p, &p->q, (size_t)p->ld)) ||
      (rc = part_alloc(p, &p->p, (size_t)p->ld)) || (rc = part_alloc(p, &p->scratch, (size_t)2 * kMaxBlocks)) ||
      (rc = part_alloc(p, &p->counter, 1)) || (rc = part_alloc(p, &p->st, 2))) {
    part_free(p);
    return rc;
  }
  p->rp = d_rp;
  cudaError_t e = cudaMemcpyAsync(d_rp, rp.data(), sizeof(int) * rp.size(), cudaMemcpyHostToDevice, p->stream);
  if (e == cudaSuccess && n_e > 0)
    e = cudaMemcpyAsync(d_D, D + e_off * n_d, sizeof(double) * n_e * n_d, cudaMemcpyHostToDevice, p->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(p->counter, 0, sizeof(unsigned), p->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(p->st, 0, 2 * sizeof(State), p->stream);
  // columns: global - (row0 - lo), so the lower halo plane starts at 0
  if (e == cudaSuccess &&
      cep_internal_fem_assemble_grid_rows(dim, nx, ny, nz, h, dt, d_D, n_d, e_off, p->row0, p->n_own, p->row0 - p->lo,
                                          d_rp, p->col, p->a, p->b, p->width, p->ld, p->ecol, p->ea, p->eb, p->dinv,
                                          p->stream))
    e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(p->stream);
  if (e != cudaSuccess) {
    part_free(p);
    return fail_msg(CEP_ERR_CUDA, "slab part assembly failed: %s", cudaGetErrorString(e));
  }
  *out = p;
  return CEP_OK;
}

int cep_part_destroy(cep_part_t p) {
  if (!p) return CEP_OK;
  part_free(p);
  return CEP_OK;
}

int cep_part_info(cep_part_t p, long *row0, long *n_own, long *plane, int *has_lo, int *has_hi) {
  if (!p) return fail_msg(CEP_ERR_ARG, "null part");
  if (row0) *row0 = (long)p->row0;
  if (n_own) *n_own = (long)p->n_own;
  if (plane) *plane = (long)p->plane;
  if (has_lo) *has_lo = p->lo > 0;
  if (has_hi) *has_hi = p->hi > 0;
  return CEP_OK;
}

int cep_part_get_csr(cep_part_t p, int *row_ptr, int *col_idx, double *a_val, double *b_val) {
  if (!p || !row_ptr || !col_idx || !a_val || !b_val) return fail_msg(CEP_ERR_ARG, "null argument");
  SLAB_CUDA(cudaMemcpyAsync(row_ptr, p->rp, sizeof(int) * (p->n_own + 1), cudaMemcpyDeviceToHost, p->stream));
  SLAB_CUDA(cudaMemcpyAsync(col_idx, p->col, sizeof(int) * p->nnz, cudaMemcpyDeviceToHost, p->stream));
  SLAB_CUDA(cudaMemcpyAsync(a_val, p->a, sizeof(double) * p->nnz, cudaMemcpyDeviceToHost, p->stream));
  SLAB_CUDA(cudaMemcpyAsync(b_val, p->b, sizeof(double) * p->nnz, cudaMemcpyDeviceToHost, p->stream));
  SLAB_CUDA(cudaStreamSynchronize(p->stream));
  const int off = (int)(p->row0 - p->lo);
  for (int64_t k = 0; k < p->nnz; ++k) col_idx[k] += off;  // back to global columns
  return CEP_OK;
}

int cep_part_set_solver(cep_part_t p, double rtol, int max_iter, int precond_norm) {
  if (!p) return fail_msg(CEP_ERR_ARG, "null part");
  if (!(rtol > 0) || max_iter < 1 || max_iter > CEP_FEM_MAX_ITER)
    return fail_msg(CEP_ERR_ARG, "rtol must be positive and max_iter in 1..%d", CEP_FEM_MAX_ITER);
  p->rtol = rtol;
  p->max_iter = max_iter;
  p->precond_norm = precond_norm ? 1 : 0;
  return CEP_OK;
}

int cep_part_pack(cep_part_t p, const void *d_v, void *d_lo, void *d_hi) {
  if (!p || !d_v) return fail_msg(CEP_ERR_ARG, "null argument");
  const double *v = static_cast<const double *>(d_v);
  const size_t bytes = sizeof(double) * (size_t)p->plane;
  if (d_lo) SLAB_CUDA(cudaMemcpyAsync(d_lo, v, bytes, cudaMemcpyDeviceToDevice, p->stream));
  if (d_hi) SLAB_CUDA(cudaMemcpyAsync(d_hi, v + (p->n_own - p->plane), bytes, cudaMemcpyDeviceToDevice, p->stream));
  return CEP_OK;
}

int cep_part_cg_begin(cep_part_t p, const void *d_v, const void *d_v_lo, const void *d_v_hi, void *d_partial) {
  if (!p || !d_v || !d_partial) return fail_msg(CEP_ERR_ARG, "null argument");
  if ((p->lo && !d_v_lo) || (p->hi && !d_v_hi)) return fail_msg(CEP_ERR_ARG, "a halo plane of V is missing");
  cep::slab::begin_kernel<<<p->nb, kBlock, 0, p->stream>>>(
      view_of(p), p->dt, p->precond_norm, static_cast<const double *>(d_v), static_cast<const double *>(d_v_lo),
      static_cast<const double *>(d_v_hi), p->x, p->r, p->z, p->p, p->st, p->scratch, p->counter,
      static_cast<double *>(d_partial));
  SLAB_CUDA(cudaGetLastError());
  return CEP_OK;
}

int cep_part_cg_direction(cep_part_t p, int iter, const void *d_all, int n_parts, void *d_send_lo, void *d_send_hi) {
  if (!p || !d_all || iter < 0) return fail_msg(CEP_ERR_ARG, "bad argument");
  if (n_parts != p->n_parts) return fail_msg(CEP_ERR_ARG, "partials of %d parts, expected %d", n_parts, p->n_parts);
  cep::slab::direction_kernel<<<p->nb, kBlock, 0, p->stream>>>(
      p->n_own, p->plane, iter, static_cast<const double *>(d_all), n_parts, p->rtol, p->max_iter, p->z, p->p, p->st,
      p->lo ? static_cast<double *>(d_send_lo) : nullptr, p->hi ? static_cast<double *>(d_send_hi) : nullptr);
  SLAB_CUDA(cudaGetLastError());
  return CEP_OK;
}

int cep_part_cg_product(cep_part_t p, int iter, const void *d_p_lo, const void *d_p_hi, void *d_partial) {
  if (!p || !d_partial || iter < 0) return fail_msg(CEP_ERR_ARG, "bad argument");
  if ((p->lo && !d_p_lo) || (p->hi && !d_p_hi)) return fail_msg(CEP_ERR_ARG, "a halo plane of p is missing");
  cep::slab::product_kernel<<<p->nb, kBlock, 0, p->stream>>>(
      view_of(p), iter, p->p, static_cast<const double *>(d_p_lo), static_cast<const double *>(d_p_hi), p->q, p->st,
      p->scratch, p->counter, static_cast<double *>(d_partial));
  SLAB_CUDA(cudaGetLastError());
  return CEP_OK;
}

int cep_part_cg_update(cep_part_t p, int iter, const void *d_all, int n_parts, void *d_partial) {
  if (!p || !d_all || !d_partial || iter < 0) return fail_msg(CEP_ERR_ARG, "bad argument");
  if (n_parts != p->n_parts) return fail_msg(CEP_ERR_ARG, "partials of %d parts, expected %d", n_parts, p->n_parts);
  cep::slab::update_kernel<<<p->nb, kBlock, 0, p->stream>>>(
      view_of(p), iter, static_cast<const double *>(d_all), n_parts, p->precond_norm, p->p, p->q, p->x, p->r, p->z,
      p->st, p->scratch, p->counter, static_cast<double *>(d_partial));
  SLAB_CUDA(cudaGetLastError());
  return CEP_OK;
}

int cep_part_cg_status(cep_part_t p, int iter, int *done, int *iters, double *res) {
  if (!p || iter < 0) return fail_msg(CEP_ERR_ARG, "bad argument");
  State s;
  SLAB_CUDA(cudaMemcpyAsync(&s, p->st + ((iter + 1) & 1), sizeof(State), cudaMemcpyDeviceToHost, p->stream));
  SLAB_CUDA(cudaStreamSynchronize(p->stream));
  if (done) *done = s.done;
  if (iters) *iters = s.conv ? s.used : -p->max_iter;
  if (res) *res = s.res;
  return CEP_OK;
}

int cep_part_cg_end(cep_part_t p, void *d_v, double t_new) {
  if (!p || !d_v) return fail_msg(CEP_ERR_ARG, "null argument");
  cep::slab::end_kernel<<<(unsigned)((p->n_own + 127) / 128), 128, 0, p->stream>>>(
      p->n_own, p->x, static_cast<double *>(d_v), p->tact, t_new, p->act_thr);
  SLAB_CUDA(cudaGetLastError());
  return CEP_OK;
}

int cep_part_bind_cells(cep_part_t p, cep_batch_t cells, const unsigned char *s1_mask, double bcl, double t_crt,
                        double dur, int n_pace, double act_thr) {
  if (!p || !cells) return fail_msg(CEP_ERR_ARG, "null argument");
  int n = 0, ns = 0;
  if (int rc = cep_batch_size(cells, &n, &ns)) return rc;
  if (n != p->n_own) return fail_msg(CEP_ERR_ARG, "the batch has %d instances, the part %lld rows", n, (long long)p->n_own);
  if (cep_internal_batch_stream(cells) != (void *)p->stream)
    return fail_msg(CEP_ERR_ARG, "the batch and the part must share one stream");
  if (!(bcl > 0) || !(dur >= 0) || n_pace < 0) return fail_msg(CEP_ERR_ARG, "bad stimulus protocol");
  if (int rc = cep_internal_batch_tissue_begin(cells, p->dt)) return rc;
  int rc;
  if (!p->mask && (rc = part_alloc(p, &p->mask, (size_t)p->n_own))) return rc;
  if (!p->tact && (rc = part_alloc(p, &p->tact, (size_t)p->n_own))) return rc;
  if (s1_mask)
    SLAB_CUDA(cudaMemcpyAsync(p->mask, s1_mask, (size_t)p->n_own, cudaMemcpyHostToDevice, p->stream));
  else
    SLAB_CUDA(cudaMemsetAsync(p->mask, 0, (size_t)p->n_own, p->stream));
  cep::slab::fill_kernel<<<(unsigned)((p->n_own + 127) / 128), 128, 0, p->stream>>>(p->n_own, p->tact, -1.0);
  SLAB_CUDA(cudaGetLastError());
  SLAB_CUDA(cudaStreamSynchronize(p->stream));
  p->cells = cells;
  p->bcl = bcl; p->t_crt = t_crt; p->dur = dur; p->n_pace = n_pace; p->act_thr = act_thr;
  return CEP_OK;
}

int cep_part_ionic_step(cep_part_t p, double t) {
  if (!p || !p->cells) return fail_msg(CEP_ERR_STATE, "no cells bound to the part");
  return cep_internal_batch_tissue_step(p->cells, p->mask, t, p->bcl, p->t_crt, p->dur, p->n_pace, nullptr, nullptr);
}

int cep_part_get_activation(cep_part_t p, double *t_act) {
  if (!p || !t_act) return fail_msg(CEP_ERR_ARG, "null argument");
  if (!p->tact) return fail_msg(CEP_ERR_STATE, "no cells bound to the part");
  SLAB_CUDA(cudaMemcpyAsync(t_act, p->tact, sizeof(double) * p->n_own, cudaMemcpyDeviceToHost, p->stream));
  SLAB_CUDA(cudaStreamSynchronize(p->stream));
  return CEP_OK;
}

}  // extern "C"
