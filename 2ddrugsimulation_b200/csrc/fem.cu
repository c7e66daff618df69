// Monodomain diffusion solve and the tissue driver: the cep_fem_* and
// cep_tissue_* C ABI (include/cep_b200.h).
//
// Replaces Cfem::solve_Bmat (fem.cpp:705-718) with PETSc KSPCG + PCJACOBI
// (fem.cpp:753-760) and the Godunov loop of Cheart::processing
// (heart.cpp:127-165, 274-430).
//
// One solve is ONE cooperative persistent launch:
//   phase 0   b = B V* / dt (the RHS build fused with the first residual),
//             r = b, z = D^-1 r, p_0 = 0, partial sums of r.z and |z|^2
//   per CG iteration (two grid barriers):
//     A   p_k = z + beta p_{k-1} evaluated on the fly inside the SpMV,
//         q = A p_k, partial p.q                             -> barrier
//     B   r -= alpha q, z = D^-1 r, partial r.z and |z|^2  -> barrier
//   (x += alpha_k p_k is applied by pass A of iteration k+1, which reads
//   p_k anyway, or by a last pass after the final iteration)
// Dots are FP64 and deterministic: every block writes one partial per
// reduction and every block sums all partials in the same fixed order, so
// each block holds bit-identical scalars and takes the same branch. x is
// written straight into the caller's V vector (x0 = 0 is implicit), so the
// solve works in place on the ionic state's V row.
//
// HBM layout of an operator with n rows (ld = n rounded up to 32):
//   CSR    row_ptr[n+1] i32, col[nnz] i32, a[nnz] f64, b[nnz] f64
//   ELL    col[width][ld] i32, a[width][ld] f64, b[width][ld] f64 (padding
//          entries point at the row itself with weight 0)
//   STENCIL a[slots][ld] f64, b[slots][ld] f64 (implicit columns)
//   CLASSED class[ld] i32, a/b [classes][slots + 1] f64
//   dinv[ld], r[ld], q[ld] f64; p0, p1, z [guard + ld + guard] f64 (guard =
//   one plane + one line + one node for grid operators, zeros); partials
//   [3][grid] f64
//
// The grid barrier spins with an iteration limit; a barrier that runs out
// sets an error word, every block leaves at its next barrier, and the host
// reports CEP_ERR_TIMEOUT.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/cep_b200.h"
#include "internal.h"

extern "C" int cep_internal_fem_assemble_grid(int dim, int nx, int ny, int nz, double h, double dt, const double *d_D,
                                              int n_d, const int *d_rp, int *d_col, double *d_a, double *d_b,
                                              int width, int64_t ld, int *d_ecol, double *d_ea, double *d_eb,
                                              double *d_dinv, void *stream);

extern "C" int cep_internal_fem_assemble_tet(int n_nodes, const double *d_xyz, const int *d_conn, const double *d_D,
                                             int n_d, double dt, const int *d_inc_ptr, const int *d_inc,
                                             const int *d_rp, const int *d_col, double *d_a, double *d_b,
                                             void *stream);

namespace {

// A copy on the object's own stream, finished before returning. A plain
// cudaMemcpy runs on the legacy stream, which a non-blocking stream does
// not wait for, and returns before a pageable upload has landed.
inline cudaError_t copy_sync(void *dst, const void *src, size_t bytes, cudaMemcpyKind kind, cudaStream_t s) {
  cudaError_t e = cudaMemcpyAsync(dst, src, bytes, kind, s);
  return e == cudaSuccess ? cudaStreamSynchronize(s) : e;
}

#define FEM_CUDA(call)                                                                                   \
  do {                                                                                                   \
    cudaError_t e_ = (call);                                                                             \
    if (e_ != cudaSuccess) {                                                                             \
      std::string m_ = std::string(#call) + ": " + cudaGetErrorString(e_);                               \
      return cep_internal_set_fail(CEP_ERR_CUDA, m_.c_str());                                            \
    }                                                                                                    \
  } while (0)

int fail_msg(int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  return cep_internal_set_fail(code, buf);
}

constexpr int kPcgBlock = 1024;
constexpr long kSpinLimit = 1L << 22;  // polls of ~0.3-0.5 us: about a second or two

}  // namespace

namespace cep {
namespace fem {

struct Status {
  int last_iters;           // iterations of the last solve (negative: hit max_iter)
  int not_converged;        // solves that hit max_iter
  long long total_iters;    // over all solves
  long long solves;
  double last_res;          // relative residual of the last solve
};

struct Ctl {
  unsigned count;  // grid barrier arrivals (bit 31: a wait ran out)
  unsigned pad0;
  int err;         // barrier timeout, for the host
  int pad;
};

// The CG direction p_k = z_{k-1} + beta p_{k-1} of a neighbour, formed on
// the fly from the previous direction and preconditioned residual (each in
// its own array, written whole by one pass: no partial-sector writes).
struct Dir {
  const double *p, *z;
  double beta;
  __device__ __forceinline__ double operator()(int64_t j) const { return fma(beta, p[j], z[j]); }
};

// Bulk L2 prefetch of [p, p + bytes) (16-byte aligned, multiple of 16).
__device__ __forceinline__ void prefetch_l2(const void *p, unsigned bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

struct CsrView {
  const int *rp, *col;
  const double *a, *b;
  template <class X>
  __device__ __forceinline__ double apply(const double *val, int64_t i, X x) const {
    double s = 0.0;
    const int e = rp[i + 1];
    for (int k = rp[i]; k < e; ++k) s = fma(val[k], x(col[k]), s);
    return s;
  }
  __device__ __forceinline__ double apply_dir(const double *val, int64_t i, const Dir &d) const {
    return apply(val, i, [&](int j) { return d(j); });
  }
  // a per-row key the product pass may load a trip ahead (none here)
  __device__ __forceinline__ int row_key(int64_t) const { return 0; }
  __device__ __forceinline__ double apply_dir_key(const double *val, int64_t i, int, const Dir &d) const {
    return apply_dir(val, i, d);
  }
  __device__ __forceinline__ void prefetch(int64_t, int64_t, int64_t, const Dir &) const {}
};

struct EllView {
  const int *col;
  const double *a, *b;
  int width;
  int64_t ld;
  template <class X>
  __device__ __forceinline__ double apply(const double *val, int64_t i, X x) const {
    double s = 0.0;
#pragma unroll 9
    for (int k = 0; k < width; ++k) s = fma(val[k * ld + i], x(col[k * ld + i]), s);
    return s;
  }
  __device__ __forceinline__ double apply_dir(const double *val, int64_t i, const Dir &d) const {
    return apply(val, i, [&](int j) { return d(j); });
  }
  __device__ __forceinline__ int row_key(int64_t) const { return 0; }
  __device__ __forceinline__ double apply_dir_key(const double *val, int64_t i, int, const Dir &d) const {
    return apply_dir(val, i, d);
  }
  __device__ __forceinline__ void prefetch(int64_t, int64_t, int64_t, const Dir &) const {}
};

// Structured-grid operator with implicit columns: slot (dk+1)*9 + (dj+1)*3 +
// (di+1) of row i couples node i with node i + di + nx*(dj + ny*dk); slots
// outside the grid hold 0 and read the row's own entry. Slots run in
// ascending column order, so a row sums its nonzeros in the same order as
// CSR/ELL. Vector gathers are unit-stride across a warp.
template <int DIM>
struct StencilView {
  const double *a, *b;  // [slots][ld]
  int nx, ny, nz;
  int64_t ld;
  template <class X>
  __device__ __forceinline__ double apply(const double *val, int64_t i, X x) const {
    const int ii = (int)i, plane = nx * ny;
    const int ix = ii % nx;
    const int iy = (ii / nx) % ny;
    const int iz = DIM == 3 ? ii / plane : 0;
    double s = 0.0;
#pragma unroll
    for (int dk = (DIM == 3 ? -1 : 0); dk <= (DIM == 3 ? 1 : 0); ++dk)
#pragma unroll
      for (int dj = -1; dj <= 1; ++dj)
#pragma unroll
        for (int di = -1; di <= 1; ++di) {
          const int slot = (DIM == 3 ? (dk + 1) * 9 : 0) + (dj + 1) * 3 + (di + 1);
          const bool in = (unsigned)(ix + di) < (unsigned)nx && (unsigned)(iy + dj) < (unsigned)ny &&
                          (DIM == 2 || (unsigned)(iz + dk) < (unsigned)nz);
          const int j = in ? ii + di + nx * dj + plane * dk : ii;
          s = fma(val[slot * ld + i], x(j), s);
        }
    return s;
  }
  // Unchecked gathers: a slot outside the grid has weight 0 and reads a
  // finite value (a wrapped neighbour, or a zero guard row before row 0 /
  // after row n-1), adding a zero as the checked form does.
  __device__ __forceinline__ double apply_dir(const double *val, int64_t i, const Dir &d) const {
    const int plane = nx * ny;
    double s = 0.0;
#pragma unroll
    for (int dk = (DIM == 3 ? -1 : 0); dk <= (DIM == 3 ? 1 : 0); ++dk)
#pragma unroll
      for (int dj = -1; dj <= 1; ++dj) {
        const int64_t row = i + (nx * dj + plane * dk);
#pragma unroll
        for (int di = -1; di <= 1; ++di) {
          const int slot = (DIM == 3 ? (dk + 1) * 9 : 0) + (dj + 1) * 3 + (di + 1);
          s = fma(val[slot * ld + i], d(row + di), s);
        }
      }
    return s;
  }
  __device__ __forceinline__ int row_key(int64_t) const { return 0; }
  __device__ __forceinline__ double apply_dir_key(const double *val, int64_t i, int, const Dir &d) const {
    return apply_dir(val, i, d);
  }
  // Rows [b, b + count) come next: fetch into L2 what the sweep has not
  // touched yet, the leading plane (3D) or line (2D) of their
  // neighbourhood (rounded out to 16-byte boundaries).
  __device__ __forceinline__ void prefetch(int64_t b, int64_t count, int64_t ld_rows, const Dir &d) const {
    const int64_t lead = DIM == 3 ? (int64_t)nx * ny : nx;
    int64_t lo = (b + lead - nx - 2) & ~(int64_t)1, hi = (b + count + lead + nx + 2) & ~(int64_t)1;
    if (hi > ld_rows) hi = ld_rows;
    if (lo < hi) {
      prefetch_l2(d.p + lo, (unsigned)((hi - lo) * sizeof(double)));
      prefetch_l2(d.z + lo, (unsigned)((hi - lo) * sizeof(double)));
    }
  }
};

// Grid operator whose rows are grouped into classes of identical
// coefficients (a uniform sheet has 9 classes; a slab whose conductivity
// varies only with depth has a few per plane): each row stores a class
// index, the coefficients live once per class in a table that stays in
// cache, so an SpMV row reads 4 bytes of matrix instead of 8 per slot.
// Slots and columns as StencilView, so each row's sum is bit-identical.
template <int DIM>
struct ClassView {
  // class rows padded to an even slot count for 16-byte coefficient loads
  static constexpr int kSlots = DIM == 3 ? 27 : 9, kStride = kSlots + 1;
  const int *cls;
  const double *a, *b;  // [classes][kStride]
  int nx, ny, nz;
  template <class X>
  __device__ __forceinline__ double apply(const double *val, int64_t i, X x) const {
    const int ii = (int)i, plane = nx * ny;
    const int ix = ii % nx;
    const int iy = (ii / nx) % ny;
    const int iz = DIM == 3 ? ii / plane : 0;
    const double *c = val + (int64_t)__ldg(cls + i) * kStride;
    double s = 0.0;
#pragma unroll
    for (int dk = (DIM == 3 ? -1 : 0); dk <= (DIM == 3 ? 1 : 0); ++dk)
#pragma unroll
      for (int dj = -1; dj <= 1; ++dj)
#pragma unroll
        for (int di = -1; di <= 1; ++di) {
          const int slot = (DIM == 3 ? (dk + 1) * 9 : 0) + (dj + 1) * 3 + (di + 1);
          const bool in = (unsigned)(ix + di) < (unsigned)nx && (unsigned)(iy + dj) < (unsigned)ny &&
                          (DIM == 2 || (unsigned)(iz + dk) < (unsigned)nz);
          const int j = in ? ii + di + nx * dj + plane * dk : ii;
          s = fma(__ldg(c + slot), x(j), s);
        }
    return s;
  }
  // Unchecked gathers as StencilView::apply_dir; coefficients two at a time.
  __device__ __forceinline__ double apply_dir(const double *val, int64_t i, const Dir &d) const {
    return apply_dir_key(val, i, __ldg(cls + i), d);
  }
  // the row's class, loaded a trip ahead by the product pass
  __device__ __forceinline__ int row_key(int64_t i) const { return __ldg(cls + i); }
  __device__ __forceinline__ double apply_dir_key(const double *val, int64_t i, int key, const Dir &d) const {
    const double2 *c2 = reinterpret_cast<const double2 *>(val + (int64_t)key * kStride);
    const int plane = nx * ny;
    double s = 0.0;
    double2 cp = make_double2(0.0, 0.0);
#pragma unroll
    for (int dk = (DIM == 3 ? -1 : 0); dk <= (DIM == 3 ? 1 : 0); ++dk)
#pragma unroll
      for (int dj = -1; dj <= 1; ++dj) {
        const int64_t row = i + (nx * dj + plane * dk);
#pragma unroll
        for (int di = -1; di <= 1; ++di) {
          const int slot = (DIM == 3 ? (dk + 1) * 9 : 0) + (dj + 1) * 3 + (di + 1);
          if ((slot & 1) == 0) cp = __ldg(c2 + (slot >> 1));
          s = fma((slot & 1) ? cp.y : cp.x, d(row + di), s);
        }
      }
    return s;
  }
  __device__ __forceinline__ void prefetch(int64_t b, int64_t count, int64_t ld_rows, const Dir &d) const {
    const int64_t lead = DIM == 3 ? (int64_t)nx * ny : nx;
    int64_t lo = (b + lead - nx - 2) & ~(int64_t)1, hi = (b + count + lead + nx + 2) & ~(int64_t)1;
    if (hi > ld_rows) hi = ld_rows;
    if (lo < hi) {
      prefetch_l2(d.p + lo, (unsigned)((hi - lo) * sizeof(double)));
      prefetch_l2(d.z + lo, (unsigned)((hi - lo) * sizeof(double)));
    }
    const int64_t ce = b + count < ld_rows ? b + count : ld_rows;
    if (b < ce) prefetch_l2(cls + b, (unsigned)((ce - b) * sizeof(int)));
  }
};

struct PcgArgs {
  int64_t n;
  double dt, rtol;
  int max_iter, precond_norm;
  double *v;  // in: V*, out: V
  const double *dinv;
  int64_t ld;          // rows allocated in each vector (n rounded up to 32)
  double *r, *q;
  double *p0, *p1, *z;  // grid formats read guard rows around [0, n) of these
  double *part;  // [3][blocks]
  Ctl *ctl;
  Status *st;
  double *tact;  // activation times (may be null)
  double t_new, act_thr;
};

__device__ __forceinline__ unsigned ld_acquire(const unsigned *p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ int ld_volatile(const int *p) { return *(const volatile int *)p; }

// Grid-wide barrier over co-resident blocks (cooperative launch), bounded.
// The arrival counter only grows within a launch (zeroed before it): the
// e-th barrier is complete once it reaches e * gridDim.x, so each block
// makes one acquire-release atomic and the last arriver needs no second
// write. A block whose wait runs out of its spin limit sets the poison bit
// in the counter (and the error word the host reads); every block sees it
// at its next arrival or poll and leaves.
constexpr unsigned kPoison = 0x80000000u;

// Test hooks of the bounded waits (cep_fem_set_wait_test): a smaller spin
// limit for every grid barrier on this device (0 = kSpinLimit) and a
// bounded sleep of block 0 before its first barrier, so that a test can make
// the other blocks' waits run out without any fault.
__device__ long long g_spin_limit_test = 0;
__device__ unsigned g_block0_delay_ns = 0;

__device__ __forceinline__ void test_delay_block0() {
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    const unsigned d = g_block0_delay_ns;
    for (unsigned t = 0; t < d; t += 1024u) __nanosleep(1024u);
  }
}

__device__ __forceinline__ unsigned atom_add_acq_rel(unsigned *p, unsigned v) {
  unsigned old;
  asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
  return old;
}

__device__ __forceinline__ bool grid_sync(Ctl *ctl, unsigned &epoch) {
  __shared__ int s_ok;
  __syncthreads();
  ++epoch;
  if (threadIdx.x == 0) {
    int ok = 1;
    const unsigned target = epoch * gridDim.x;
    const unsigned old = atom_add_acq_rel(&ctl->count, 1u);
    if (old & kPoison) {
      ok = 0;
    } else if (old + 1u < target) {
      const long long lim = g_spin_limit_test > 0 ? g_spin_limit_test : (long long)kSpinLimit;
      long long spins = 0;
      for (;;) {
        const unsigned c = ld_acquire(&ctl->count);
        if (c & kPoison) {
          ok = 0;
          break;
        }
        if (c >= target) break;
        if (++spins > lim) {
          atomicOr(&ctl->count, kPoison);
          atomicExch(&ctl->err, 1);
          ok = 0;
          break;
        }
      }
    }
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// Fixed-order block reduction of two values; thread 0 gets the sums.
__device__ __forceinline__ void block_sum2(double &x, double &y) {
  constexpr int kWarps = kPcgBlock / 32;
  __shared__ double sx[kWarps], sy[kWarps];
  for (int o = 16; o > 0; o >>= 1) {
    x += __shfl_down_sync(0xffffffffu, x, o);
    y += __shfl_down_sync(0xffffffffu, y, o);
  }
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) {
    sx[w] = x;
    sy[w] = y;
  }
  __syncthreads();
  if (w == 0) {
    x = l < kWarps ? sx[l] : 0.0;
    y = l < kWarps ? sy[l] : 0.0;
    for (int o = 16; o > 0; o >>= 1) {
      x += __shfl_down_sync(0xffffffffu, x, o);
      y += __shfl_down_sync(0xffffffffu, y, o);
    }
  }
  __syncthreads();
}

// Several independent operators of one format in one cooperative launch
// (tissues of a batch: concentrations, requests): the grid is split into
// contiguous block ranges, one per operator in proportion to its rows; each
// operator runs its own Jacobi-PCG with its own scalars and stopping test
// while all share the grid barriers, so the barrier latency is paid once
// per iteration for the whole batch. An operator that has converged idles
// through the barriers until the last one is done.
template <class M>
struct PcgOp {
  M m;
  PcgArgs a;       // a.part holds 3 * nblocks partials, a.ctl unused
  int block0, nblocks;
};

// The operators of a batched launch travel as a kernel parameter, so each
// block reads its operator's fields from the constant bank on use instead
// of holding a copy in registers.
constexpr int kMaxGroup = 64;
template <class M>
struct PcgOps {
  PcgOp<M> op[kMaxGroup];
};

__device__ __forceinline__ void range_total2(const double *pa, const double *pb, int nb, double &a, double &b) {
  __shared__ double s[2];
  if (threadIdx.x < 32) {
    constexpr int kU = 8;
    double x = 0.0, y = 0.0;
    for (int base = 0; base < nb; base += 32 * kU) {
      double xs[kU], ys[kU];
#pragma unroll
      for (int u = 0; u < kU; ++u) {
        const int k = base + u * 32 + threadIdx.x;
        xs[u] = k < nb ? __ldcg(pa + k) : 0.0;
        ys[u] = (pb && k < nb) ? __ldcg(pb + k) : 0.0;
      }
#pragma unroll
      for (int u = 0; u < kU; ++u) {
        x += xs[u];
        y += ys[u];
      }
    }
    for (int o = 16; o > 0; o >>= 1) {
      x += __shfl_down_sync(0xffffffffu, x, o);
      y += __shfl_down_sync(0xffffffffu, y, o);
    }
    if (threadIdx.x == 0) {
      s[0] = x;
      s[1] = y;
    }
  }
  __syncthreads();
  a = s[0];
  b = s[1];
  __syncthreads();
}

// Jacobi-PCG of one operator on block lb of the NB blocks it owns (the
// whole grid for a single solve, a contiguous range of a batched launch).
// Each thread takes rows two at a time (i and i + stride, the second
// clamped to a valid row and masked) so both rows' gathers are in flight;
// its partial sums still add rows in increasing order. In a batched launch
// (n_ops > 1) an operator that has converged keeps taking the grid barriers
// until every operator has, counted in ops_done.
//
// Vectors: r, q, z, the caller's V (x), and two direction buffers used in
// turn. Iteration k: pass A reads p_{k-1} and z_{k-1} around each row,
// forms p_k into the other buffer, writes q = A p_k and applies the
// previous iteration's x update; pass B updates r and writes z_k.
template <class M>
__device__ __forceinline__ void pcg_body(const M &m, const PcgArgs &a, int NB, int lb, Ctl *ctl, int *ops_done,
                                         int n_ops, double t_new) {
  const bool lead = lb == 0 && threadIdx.x == 0;
  const int64_t stride = (int64_t)NB * kPcgBlock;
  const int64_t i0 = (int64_t)lb * kPcgBlock + threadIdx.x;
  double *part0 = a.part, *part1 = a.part + NB, *part2 = a.part + 2 * NB;
  const double *v_in = a.v;
  unsigned epoch = 0;  // grid barriers passed
  // phase 0: b = B V / dt, r = b, z = D^-1 b, p_0 = 0
  double s0 = 0.0, s1 = 0.0;
  for (int64_t i = i0; i < a.n; i += 2 * stride) {
    const bool two = i + stride < a.n;
    const int64_t i2 = two ? i + stride : i;
    const double b1 = m.apply(m.b, i, [&](int j) { return v_in[j]; }) / a.dt;
    const double b2 = m.apply(m.b, i2, [&](int j) { return v_in[j]; }) / a.dt;
    const double z1 = a.dinv[i] * b1, z2 = a.dinv[i2] * b2;
    a.r[i] = b1;
    a.z[i] = z1;
    a.p0[i] = 0.0;
    s0 = fma(b1, z1, s0);
    s1 = a.precond_norm ? fma(z1, z1, s1) : fma(b1, b1, s1);
    if (two) {
      a.r[i2] = b2;
      a.z[i2] = z2;
      a.p0[i2] = 0.0;
      s0 = fma(b2, z2, s0);
      s1 = a.precond_norm ? fma(z2, z2, s1) : fma(b2, b2, s1);
    }
  }
  block_sum2(s0, s1);
  if (threadIdx.x == 0) {
    part0[lb] = s0;
    part1[lb] = s1;
  }
  if (!grid_sync(ctl, epoch)) return;
  double rz, nn0;
  range_total2(part0, part1, NB, rz, nn0);
  const double n0 = sqrt(nn0);
  int used = 0;
  double res = n0 > 0.0 ? 1.0 : 0.0;
  bool conv = false, done = false, counted = false;
  if (n0 == 0.0) {
    for (int64_t i = i0; i < a.n; i += stride) a.v[i] = 0.0;
    conv = done = true;
  }
  double *pc = a.p0, *pn = a.p1;
  double beta = 0.0;  // p_1 = z_0 + 0 * p_0
  double alpha_prev = 0.0;
  for (int it = 1; !(n_ops == 1 && done); ++it) {
    // A: p_k and q = A p_k (operators still iterating); report completions
    if (!done) {
      double spq = 0.0, unused = 0.0;
      int key1 = 0, key2 = 0;  // this trip's row keys (the classed format's class index)
      if (i0 < a.n) {
        key1 = m.row_key(i0);
        key2 = m.row_key(i0 + stride < a.n ? i0 + stride : i0);
      }
      for (int64_t i = i0; i < a.n; i += 2 * stride) {
        // the block's rows two trips ahead, fetched into L2 by one thread
        const Dir d{pc, a.z, beta};
        if (threadIdx.x == 0) {
          const int64_t nb = i + 2 * stride;
          m.prefetch(nb, kPcgBlock, a.ld, d);
          m.prefetch(nb + stride, kPcgBlock, a.ld, d);
        }
        const bool two = i + stride < a.n;
        const int64_t i2 = two ? i + stride : i;
        // next trip's keys, in flight while this trip computes
        const int64_t j1 = i + 2 * stride, j2 = j1 + stride < a.n ? j1 + stride : j1;
        const int nkey1 = j1 < a.n ? m.row_key(j1) : 0, nkey2 = j1 < a.n ? m.row_key(j2) : 0;
        const double q1 = m.apply_dir_key(m.a, i, key1, d);
        const double q2 = m.apply_dir_key(m.a, i2, key2, d);
        key1 = nkey1;
        key2 = nkey2;
        const double c1 = pc[i], c2 = pc[i2];
        const double p1 = fma(beta, c1, a.z[i]), p2 = fma(beta, c2, a.z[i2]);
        pn[i] = p1;
        a.q[i] = q1;
        spq = fma(p1, q1, spq);
        // x_{k-1} += alpha_{k-1} p_{k-1}, deferred from the last iteration
        if (it > 1) a.v[i] = it == 2 ? alpha_prev * c1 : fma(alpha_prev, c1, a.v[i]);
        if (two) {
          pn[i2] = p2;
          a.q[i2] = q2;
          spq = fma(p2, q2, spq);
          if (it > 1) a.v[i2] = it == 2 ? alpha_prev * c2 : fma(alpha_prev, c2, a.v[i2]);
        }
      }
      block_sum2(spq, unused);
      if (threadIdx.x == 0) part2[lb] = spq;
    } else if (!counted) {
      if (lead) atomicAdd(ops_done, 1);
      counted = true;
    }
    if (!grid_sync(ctl, epoch)) return;
    if (n_ops > 1) {
      if (ld_volatile(ops_done) == n_ops) break;  // every block reads the same count here
      if (done) {
        if (!grid_sync(ctl, epoch)) return;
        continue;
      }
    }
    double pq, dummy;
    range_total2(part2, nullptr, NB, pq, dummy);
    const double alpha = rz / pq;
    double *t = pc;  // pn now holds p_k
    pc = pn;
    pn = t;
    // B: r -= alpha q, z = D^-1 r (x += alpha p rides on the next pass A)
    double srz = 0.0, snr = 0.0;
    for (int64_t i = i0; i < a.n; i += 2 * stride) {
      const bool two = i + stride < a.n;
      const int64_t i2 = two ? i + stride : i;
      const double ra = fma(-alpha, a.q[i], a.r[i]), rb = fma(-alpha, a.q[i2], a.r[i2]);
      const double za = a.dinv[i] * ra, zb = a.dinv[i2] * rb;
      a.r[i] = ra;
      a.z[i] = za;
      srz = fma(ra, za, srz);
      snr = a.precond_norm ? fma(za, za, snr) : fma(ra, ra, snr);
      if (two) {
        a.r[i2] = rb;
        a.z[i2] = zb;
        srz = fma(rb, zb, srz);
        snr = a.precond_norm ? fma(zb, zb, snr) : fma(rb, rb, snr);
      }
    }
    block_sum2(srz, snr);
    if (threadIdx.x == 0) {
      part0[lb] = srz;
      part1[lb] = snr;
    }
    if (!grid_sync(ctl, epoch)) return;
    double rz_new, nr2;
    range_total2(part0, part1, NB, rz_new, nr2);
    const double nr = sqrt(nr2);
    res = nr / n0;
    used = it;
    if (nr <= a.rtol * n0) {
      conv = done = true;
    } else if (it >= a.max_iter) {
      done = true;
    }
    alpha_prev = alpha;
    if (done)  // the last iteration's x update: no pass A follows
      for (int64_t i = i0; i < a.n; i += stride) {
        a.v[i] = it == 1 ? alpha * pc[i] : fma(alpha, pc[i], a.v[i]);
      }
    beta = rz_new / rz;
    rz = rz_new;
  }
  if (a.tact)
    for (int64_t i = i0; i < a.n; i += stride)
      if (a.tact[i] < 0.0 && a.v[i] >= a.act_thr) a.tact[i] = t_new;
  if (lead) {
    a.st->last_iters = conv ? used : -a.max_iter;
    a.st->last_res = res;
    a.st->total_iters += conv ? used : a.max_iter;
    a.st->solves += 1;
    if (!conv) a.st->not_converged += 1;
  }
}

// One operator over the whole cooperative grid.
template <class M>
__global__ void __launch_bounds__(kPcgBlock) pcg_kernel(const __grid_constant__ M m,
                                                        const __grid_constant__ PcgArgs a) {
  test_delay_block0();
  pcg_body(m, a, (int)gridDim.x, (int)blockIdx.x, a.ctl, nullptr, 1, a.t_new);
}

// Several operators, each on its own block range (see PcgOp).
template <class M>
__global__ void __launch_bounds__(kPcgBlock) pcg_many_kernel(const __grid_constant__ PcgOps<M> ops, int n_ops,
                                                             Ctl *ctl, int *ops_done) {
  test_delay_block0();
  int o = 0;
  while (o + 1 < n_ops && (int)blockIdx.x >= ops.op[o + 1].block0) ++o;
  const PcgOp<M> &op = ops.op[o];
  pcg_body(op.m, op.a, op.nblocks, (int)blockIdx.x - op.block0, ctl, ops_done, n_ops, op.a.t_new);
}

// y = A x or B x (tests)
template <class M>
__global__ void spmv_kernel(M m, int which, int64_t n, const double *x, double *y) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  y[i] = m.apply(which ? m.b : m.a, i, [&](int j) { return x[j]; });
}

// A smooth membrane-potential-like field for the format autotuner.
__global__ void smooth_field_kernel(int64_t n, double *v) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) v[i] = -40.0 + 45.0 * sin(1e-3 * (double)i);
}

__global__ void csr_to_ell_kernel(int64_t n, const int *rp, const int *col, const double *a, const double *b,
                                  int width, int64_t ld, int *ecol, double *ea, double *eb, double *dinv) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int slot = 0;
  double diag = 1.0;
  for (int k = rp[i]; k < rp[i + 1]; ++k, ++slot) {
    ecol[slot * ld + i] = col[k];
    ea[slot * ld + i] = a[k];
    eb[slot * ld + i] = b[k];
    if (col[k] == i) diag = a[k];
  }
  for (; slot < width; ++slot) {
    ecol[slot * ld + i] = (int)i;
    ea[slot * ld + i] = 0.0;
    eb[slot * ld + i] = 0.0;
  }
  dinv[i] = 1.0 / diag;
}

__global__ void csr_to_stencil_kernel(int64_t n, int nx, int ny, int dim, const int *rp, const int *col,
                                      const double *a, const double *b, int64_t ld, double *sa, double *sb) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int slots = dim == 3 ? 27 : 9;
  for (int k = 0; k < slots; ++k) {
    sa[k * ld + i] = 0.0;
    sb[k * ld + i] = 0.0;
  }
  const int64_t plane = (int64_t)nx * ny;
  const int ix = (int)(i % nx), iy = (int)((i / nx) % ny), iz = (int)(i / plane);
  for (int k = rp[i]; k < rp[i + 1]; ++k) {
    const int64_t j = col[k];
    const int jx = (int)(j % nx), jy = (int)((j / nx) % ny), jz = (int)(j / plane);
    const int slot = (dim == 3 ? (jz - iz + 1) * 9 : 0) + (jy - iy + 1) * 3 + (jx - ix + 1);
    sa[slot * ld + i] = a[k];
    sb[slot * ld + i] = b[k];
  }
}

}  // namespace fem
}  // namespace cep

using namespace cep::fem;

struct cep_fem {
  int n = 0;
  int64_t ld = 0, nnz = 0;
  int width = 0, format = CEP_FEM_ELL;
  double dt = 0.0;
  cudaStream_t stream = nullptr;
  int *rp = nullptr, *col = nullptr, *ecol = nullptr;
  double *a = nullptr, *b = nullptr, *ea = nullptr, *eb = nullptr, *dinv = nullptr;
  double *sa = nullptr, *sb = nullptr;  // stencil values (grid operators only)
  int *cls = nullptr;                   // row classes (grid operators with few distinct rows)
  double *ca = nullptr, *cb = nullptr;  // [classes][slots]
  int n_classes = 0;
  int dim = 0, gnx = 0, gny = 0, gnz = 0;
  double *r = nullptr, *q = nullptr, *part = nullptr;
  double *D = nullptr;  // grid operators: conductivity per element [n_elem][n_d] (pseudo-ECG)
  int n_d = 0;
  double h = 0.0;
  double *p0 = nullptr, *p1 = nullptr, *z = nullptr;  // row 0 of [guard | ld | guard] zero-filled buffers
  int64_t guard = 0;  // rows a grid-format gather may reach past either end
  Ctl *ctl = nullptr;
  Status *st = nullptr;
  int grid = 0;
  double rtol = 1e-5;  // PETSc's default KSP rtol (the reference sets none)
  int max_iter = 10000;
  int precond_norm = 1;
  std::vector<void *> allocs;
};

namespace {

template <class T>
int fem_alloc(cep_fem *f, T **p, size_t count) {
  void *q = nullptr;
  const cudaError_t e = cudaMalloc(&q, count * sizeof(T) + 256);
  if (e != cudaSuccess) return fail_msg(CEP_ERR_OOM, "cudaMalloc(%zu bytes): %s", count * sizeof(T), cudaGetErrorString(e));
  f->allocs.push_back(q);
  *p = static_cast<T *>(q);
  return CEP_OK;
}

void fem_free(cep_fem *f) {
  for (void *p : f->allocs) cudaFree(p);
  delete f;
}

CsrView csr_view(const cep_fem *f) { return CsrView{f->rp, f->col, f->a, f->b}; }
EllView ell_view(const cep_fem *f) { return EllView{f->ecol, f->ea, f->eb, f->width, f->ld}; }
template <int D>
StencilView<D> stencil_view(const cep_fem *f) {
  return StencilView<D>{f->sa, f->sb, f->gnx, f->gny, f->gnz, f->ld};
}

template <int D>
ClassView<D> class_view(const cep_fem *f) {
  return ClassView<D>{f->cls, f->ca, f->cb, f->gnx, f->gny, f->gnz};
}

// Dispatch a functor on the operator's current format view.
template <class Fn>
auto with_view(const cep_fem *f, Fn fn) {
  if (f->format == CEP_FEM_CSR) return fn(csr_view(f));
  if (f->format == CEP_FEM_STENCIL) return f->dim == 3 ? fn(stencil_view<3>(f)) : fn(stencil_view<2>(f));
  if (f->format == CEP_FEM_CLASSED) return f->dim == 3 ? fn(class_view<3>(f)) : fn(class_view<2>(f));
  return fn(ell_view(f));
}

// Group identical stencil rows (A and B coefficients bit-equal) into
// classes; skipped when distinct rows exceed an eighth of the rows, where
// the index would save little.
int fem_build_classes(cep_fem *f) {
  const int slots = f->dim == 3 ? 27 : 9;
  const int64_t n = f->n, ld = f->ld;
  std::vector<double> sa((size_t)slots * ld), sb((size_t)slots * ld);
  FEM_CUDA(copy_sync(sa.data(), f->sa, sizeof(double) * sa.size(), cudaMemcpyDeviceToHost, f->stream));
  FEM_CUDA(copy_sync(sb.data(), f->sb, sizeof(double) * sb.size(), cudaMemcpyDeviceToHost, f->stream));
  std::unordered_map<uint64_t, std::vector<int>> buckets;
  std::vector<int> cls(ld, 0);
  std::vector<double> ta, tb;
  const int64_t limit = std::max<int64_t>(64, n / 8);
  const int stride = slots + 1;  // even, for 16-byte coefficient loads
  for (int64_t i = 0; i < n; ++i) {
    uint64_t hsh = 1469598103934665603ull;
    for (int k = 0; k < slots; ++k) {
      uint64_t u, w;
      std::memcpy(&u, &sa[(size_t)k * ld + i], 8);
      std::memcpy(&w, &sb[(size_t)k * ld + i], 8);
      hsh = (hsh ^ u) * 1099511628211ull;
      hsh = (hsh ^ w) * 1099511628211ull;
    }
    auto &bucket = buckets[hsh];
    int found = -1;
    for (int c : bucket) {
      bool eq = true;
      for (int k = 0; k < slots && eq; ++k)
        eq = std::memcmp(&ta[(size_t)c * stride + k], &sa[(size_t)k * ld + i], 8) == 0 &&
             std::memcmp(&tb[(size_t)c * stride + k], &sb[(size_t)k * ld + i], 8) == 0;
      if (eq) {
        found = c;
        break;
      }
    }
    if (found < 0) {
      found = (int)(ta.size() / stride);
      if (found >= limit) return CEP_OK;  // too many distinct rows: no classed form
      for (int k = 0; k < slots; ++k) {
        ta.push_back(sa[(size_t)k * ld + i]);
        tb.push_back(sb[(size_t)k * ld + i]);
      }
      ta.push_back(0.0);
      tb.push_back(0.0);
      bucket.push_back(found);
    }
    cls[i] = found;
  }
  int rc;
  if ((rc = fem_alloc(f, &f->cls, (size_t)ld)) || (rc = fem_alloc(f, &f->ca, ta.size())) ||
      (rc = fem_alloc(f, &f->cb, tb.size())))
    return rc;
  FEM_CUDA(copy_sync(f->cls, cls.data(), sizeof(int) * ld, cudaMemcpyHostToDevice, f->stream));
  FEM_CUDA(copy_sync(f->ca, ta.data(), sizeof(double) * ta.size(), cudaMemcpyHostToDevice, f->stream));
  FEM_CUDA(copy_sync(f->cb, tb.data(), sizeof(double) * tb.size(), cudaMemcpyHostToDevice, f->stream));
  f->n_classes = (int)(ta.size() / stride);
  return CEP_OK;
}

// Buffers shared by both formats, the cooperative grid size, and zeroed
// control words.
int fem_finish_setup(cep_fem *f) {
  int rc;
  const size_t ld = (size_t)f->ld;
  if ((rc = fem_alloc(f, &f->r, ld)) || (rc = fem_alloc(f, &f->q, ld))) return rc;
  // grid formats gather up to one plane + one line + one node either side
  // (rounded up to 32 rows, so an even row index is 16-byte aligned)
  f->guard = f->dim == 3 ? (int64_t)f->gnx * f->gny + f->gnx + 1 : f->dim == 2 ? (int64_t)f->gnx + 1 : 0;
  f->guard = (f->guard + 31) / 32 * 32;
  const size_t span = ld + 2 * (size_t)f->guard;
  for (double **v : {&f->p0, &f->p1, &f->z}) {
    if ((rc = fem_alloc(f, v, span))) return rc;
    FEM_CUDA(cudaMemsetAsync(*v, 0, sizeof(double) * span, f->stream));
    *v += f->guard;
  }
  int dev = 0, sms = 0, per_sm_csr = 0, per_sm_ell = 0;
  FEM_CUDA(cudaGetDevice(&dev));
  FEM_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  FEM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_csr, pcg_kernel<CsrView>, kPcgBlock, 0));
  FEM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_ell, pcg_kernel<EllView>, kPcgBlock, 0));
  int per_sm_s2 = 0, per_sm_s3 = 0;
  FEM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_s2, pcg_kernel<StencilView<2>>, kPcgBlock, 0));
  FEM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_s3, pcg_kernel<StencilView<3>>, kPcgBlock, 0));
  int per_sm_c2 = 0, per_sm_c3 = 0;
  FEM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_c2, pcg_kernel<ClassView<2>>, kPcgBlock, 0));
  FEM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_c3, pcg_kernel<ClassView<3>>, kPcgBlock, 0));
  per_sm_s2 = std::min(per_sm_s2, per_sm_c2);
  per_sm_s3 = std::min(per_sm_s3, per_sm_c3);
  // one block per SM: fewer arrivals per grid barrier and fewer partials
  if (std::min(std::min(per_sm_csr, per_sm_ell), std::min(per_sm_s2, per_sm_s3)) < 1)
    return fail_msg(CEP_ERR_CUDA, "PCG kernel does not fit on an SM");
  const int64_t need = (f->n + kPcgBlock - 1) / kPcgBlock;
  f->grid = (int)std::max<int64_t>(1, std::min<int64_t>((int64_t)sms, need));
  if ((rc = fem_alloc(f, &f->part, (size_t)3 * f->grid)) || (rc = fem_alloc(f, &f->ctl, 1)) ||
      (rc = fem_alloc(f, &f->st, 1)))
    return rc;
  FEM_CUDA(cudaMemsetAsync(f->ctl, 0, sizeof(Ctl), f->stream));
  FEM_CUDA(cudaMemsetAsync(f->st, 0, sizeof(Status), f->stream));
  FEM_CUDA(cudaStreamSynchronize(f->stream));
  return CEP_OK;
}

template <class M>
int launch_pcg(cep_fem *f, const M &m, double *v, double *tact, double t_new, double thr) {
  PcgArgs a;
  a.n = f->n;
  a.ld = f->ld;
  a.dt = f->dt;
  a.rtol = f->rtol;
  a.max_iter = f->max_iter;
  a.precond_norm = f->precond_norm;
  a.v = v;
  a.dinv = f->dinv;
  a.r = f->r; a.q = f->q; a.p0 = f->p0; a.p1 = f->p1; a.z = f->z;
  a.part = f->part;
  a.ctl = f->ctl;
  a.st = f->st;
  a.tact = tact;
  a.t_new = t_new;
  a.act_thr = thr;
  M mm = m;
  void *args[] = {&mm, &a};
  FEM_CUDA(cudaMemsetAsync(f->ctl, 0, sizeof(Ctl), f->stream));
  FEM_CUDA(cudaLaunchCooperativeKernel((const void *)pcg_kernel<M>, dim3(f->grid), dim3(kPcgBlock), args, 0,
                                       f->stream));
  return CEP_OK;
}

int fem_solve_async(cep_fem *f, double *d_v, double *tact, double t_new, double thr) {
  return with_view(f, [&](auto m) { return launch_pcg(f, m, d_v, tact, t_new, thr); });
}

int fem_check_ctl(cep_fem *f) {
  Ctl c;
  FEM_CUDA(cudaMemcpyAsync(&c, f->ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, f->stream));
  FEM_CUDA(cudaStreamSynchronize(f->stream));
  if (c.err) return fail_msg(CEP_ERR_TIMEOUT, "PCG grid barrier ran out of its spin limit");
  return CEP_OK;
}

// Time short fixed-length CG solves (8 iterations, no early stop) in each
// available format on a smooth synthetic field and keep the fastest. The
// operator's counters and solver settings are restored afterwards.
int fem_autotune(cep_fem *f) {
  double *tv = nullptr;
  FEM_CUDA(cudaMalloc(&tv, sizeof(double) * f->ld));
  Status saved;
  FEM_CUDA(copy_sync(&saved, f->st, sizeof(Status), cudaMemcpyDeviceToHost, f->stream));
  const double rtol = f->rtol;
  const int max_iter = f->max_iter;
  f->rtol = 1e-300;
  f->max_iter = 40;  // long enough that launch and barrier jitter do not decide
  cudaEvent_t e0, e1;
  FEM_CUDA(cudaEventCreate(&e0));
  FEM_CUDA(cudaEventCreate(&e1));
  float best = 1e30f;
  int best_fmt = CEP_FEM_ELL, rc = CEP_OK;
  for (int fmt : {CEP_FEM_CSR, CEP_FEM_ELL, CEP_FEM_STENCIL, CEP_FEM_CLASSED}) {
    if (fmt == CEP_FEM_STENCIL && !f->sa) continue;
    if (fmt == CEP_FEM_CLASSED && !f->cls) continue;
    f->format = fmt;
    for (int rep = 0; rep < 5 && rc == CEP_OK; ++rep) {
      smooth_field_kernel<<<(unsigned)((f->n + 255) / 256), 256, 0, f->stream>>>((int64_t)f->n, tv);
      cudaEventRecord(e0, f->stream);
      rc = fem_solve_async(f, tv, nullptr, 0.0, 0.0);
      cudaEventRecord(e1, f->stream);
      if (cudaEventSynchronize(e1) != cudaSuccess) rc = fail_msg(CEP_ERR_CUDA, "autotune solve failed");
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      if (rep >= 1 && ms < best) {
        best = ms;
        best_fmt = fmt;
      }
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  f->rtol = rtol;
  f->max_iter = max_iter;
  cudaFree(tv);
  if (rc) return rc;
  if ((rc = fem_check_ctl(f))) return rc;
  FEM_CUDA(copy_sync(f->st, &saved, sizeof(Status), cudaMemcpyHostToDevice, f->stream));
  FEM_CUDA(cudaGetLastError());
  f->format = best_fmt;
  return CEP_OK;
}

int fem_set_format(cep_fem *f, int format) {
  if (format == CEP_FEM_AUTO) return fem_autotune(f);
  if (format != CEP_FEM_CSR && format != CEP_FEM_ELL && format != CEP_FEM_STENCIL && format != CEP_FEM_CLASSED)
    return fail_msg(CEP_ERR_ARG, "unknown sparse format %d", format);
  if (format == CEP_FEM_CLASSED && !f->cls)
    return fail_msg(CEP_ERR_ARG, "the classed format needs a grid operator with few distinct rows");
  if (format == CEP_FEM_STENCIL && !f->sa)
    return fail_msg(CEP_ERR_ARG, "the stencil format needs an operator built on a structured grid");
  f->format = format;
  return CEP_OK;
}

}  // namespace

// ---------------------------------------------------------------- tissue
struct cep_tissue {
  cep_batch_t cells = nullptr;
  cep_fem_t fem = nullptr;
  cudaStream_t stream = nullptr;
  int n = 0;
  unsigned char *mask = nullptr;
  double bcl = 1000.0, t_crt = 0.0, dur = 0.0;
  int n_pace = 0;
  double *tact = nullptr;
  double act_thr = -30.0;
  double dt = 0.01, t = 0.0;
  long steps = 0;
  // pseudo-ECG: electrodes, per-block partials, records on the device
  int n_el = 0;
  double *el = nullptr, *ecg_part = nullptr, *ecg_rec = nullptr;
  long ecg_every = 1, ecg_max = 0, ecg_n = 0;
  // S1-S2 / ectopic protocol: device state, region, reset snapshot
  int proto_kind = CEP_S2_NONE;
  CepProto *proto = nullptr;
  unsigned char *mask2 = nullptr;
  int *s2_nodes = nullptr, s2_count = 0, ns = 0;
  double *s2_snap = nullptr;  // [ns][s2_count]
};

namespace {

constexpr int kEcgBlock = 256, kEcgChunk = 16;

// Pseudo-ECG of a grid tissue (Cheart::Radiate, heart.cpp:640-690): for
// each electrode x, phi = w sum_e sum_g (D_e grad V(g)) . (c_e - x) detJ /
// |c_e - x|^3, c_e the element centroid, w = 1/6 (the reference's weight),
// Gauss points +-0.57735 as the assembly. With symmetric Gauss points the
// element's sum over g of grad V is (2/h) sum_n V_n s_n (s_n = the local
// node's corner signs), so each element costs one gradient and one dot
// product per electrode. Electrodes kEcgChunk at a time; each block writes
// one partial per electrode, summed in a fixed order by ecg_sum_kernel.
template <int DIM>
__global__ void __launch_bounds__(kEcgBlock) ecg_kernel(const double *__restrict__ v, const double *__restrict__ D,
                                                        int n_d, int nx, int ny, int nz, double h,
                                                        const double *__restrict__ el, int e0, int ne,
                                                        double *__restrict__ part) {
  const int64_t n_elem = (int64_t)(nx - 1) * (ny - 1) * (DIM == 3 ? (nz - 1) : 1);
  const double inv = 2.0 / h, jac = 0.5 * h;
  const double detJ = DIM == 3 ? jac * jac * jac : jac * jac;
  constexpr int NN = DIM == 3 ? 8 : 4;
  double acc[kEcgChunk];
#pragma unroll
  for (int k = 0; k < kEcgChunk; ++k) acc[k] = 0.0;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n_elem; e += (int64_t)gridDim.x * blockDim.x) {
    const int ex = (int)(e % (nx - 1)), ey = (int)((e / (nx - 1)) % (ny - 1));
    const int ez = DIM == 3 ? (int)(e / ((int64_t)(nx - 1) * (ny - 1))) : 0;
    // sum over Gauss points of grad V, times detJ (local node order of the assembly)
    double gx = 0.0, gy = 0.0, gz = 0.0;
#pragma unroll
    for (int a = 0; a < NN; ++a) {
      const int ox = (a == 1 || a == 2 || a == 5 || a == 6) ? 1 : 0;
      const int oy = (a == 2 || a == 3 || a == 6 || a == 7) ? 1 : 0;
      const int oz = a >= 4 ? 1 : 0;
      const double va = v[(int64_t)(ex + ox) + (int64_t)nx * ((ey + oy) + (int64_t)ny * (ez + oz))];
      gx += ox ? va : -va;
      gy += oy ? va : -va;
      if (DIM == 3) gz += oz ? va : -va;
    }
    const double sc = inv * detJ;
    gx *= sc;
    gy *= sc;
    gz *= sc;
    const double *d = D + e * n_d;
    double qx, qy, qz;
    if (n_d == 1) {
      qx = d[0] * gx; qy = d[0] * gy; qz = DIM == 3 ? d[0] * gz : 0.0;
    } else if (DIM == 2) {
      qx = d[0] * gx + d[1] * gy; qy = d[1] * gx + d[2] * gy; qz = 0.0;
    } else {
      qx = d[0] * gx + d[1] * gy + d[2] * gz; qy = d[1] * gx + d[3] * gy + d[4] * gz;
      qz = d[2] * gx + d[4] * gy + d[5] * gz;
    }
    const double cx = (ex + 0.5) * h, cy = (ey + 0.5) * h, cz = DIM == 3 ? (ez + 0.5) * h : 0.0;
#pragma unroll
    for (int k = 0; k < kEcgChunk; ++k) {
      if (k < ne) {
        const double rx = cx - el[3 * (e0 + k)], ry = cy - el[3 * (e0 + k) + 1], rz = cz - el[3 * (e0 + k) + 2];
        const double rr = sqrt(rx * rx + ry * ry + rz * rz);
        acc[k] += (qx * rx + qy * ry + qz * rz) / (rr * rr * rr);
      }
    }
  }
  // fixed-order block sums, one partial per electrode and block
  __shared__ double sm[kEcgBlock / 32];
  for (int k = 0; k < ne; ++k) {
    double x = acc[k];
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = x;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int w = 0; w < kEcgBlock / 32; ++w) t += sm[w];
      part[(int64_t)(e0 + k) * gridDim.x + blockIdx.x] = t;
    }
    __syncthreads();
  }
}

__global__ void ecg_sum_kernel(const double *part, int blocks, int n_el, double w, double *rec) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n_el) return;
  double t = 0.0;
  for (int b = 0; b < blocks; ++b) t += part[(int64_t)k * blocks + b];
  rec[k] = w * t;
}

int ecg_blocks() {
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return std::max(1, 2 * sms);
}

// record the tissue's pseudo-ECG for its current V (asynchronous)
int ecg_record(cep_tissue *t) {
  if (t->n_el == 0 || t->ecg_n >= t->ecg_max || t->steps % t->ecg_every != 0) return CEP_OK;
  const cep_fem *f = t->fem;
  const int blocks = ecg_blocks();
  const double *v = cep_internal_batch_v(t->cells);
  for (int e0 = 0; e0 < t->n_el; e0 += kEcgChunk) {
    const int ne = std::min(kEcgChunk, t->n_el - e0);
    if (f->dim == 3)
      ecg_kernel<3><<<blocks, kEcgBlock, 0, t->stream>>>(v, f->D, f->n_d, f->gnx, f->gny, f->gnz, f->h, t->el, e0, ne,
                                                         t->ecg_part);
    else
      ecg_kernel<2><<<blocks, kEcgBlock, 0, t->stream>>>(v, f->D, f->n_d, f->gnx, f->gny, 1, f->h, t->el, e0, ne,
                                                         t->ecg_part);
  }
  ecg_sum_kernel<<<(t->n_el + 127) / 128, 128, 0, t->stream>>>(t->ecg_part, blocks, t->n_el, 1.0 / 6.0,
                                                                t->ecg_rec + (int64_t)t->ecg_n * t->n_el);
  FEM_CUDA(cudaGetLastError());
  ++t->ecg_n;
  return CEP_OK;
}

// The protocol trigger of one tissue before its ionic step at time t
// (Cheart::apply_s2 / apply_ectopic, heart.cpp:452-501, evaluated only in
// the last S1 pace, heart.cpp:322-323).
__global__ void proto_kernel(CepProto *p, const double *v, double t, double bcl, int n_pace) {
  p->reset_now = 0;
  if ((int)(t / bcl) != n_pace - 1) return;
  const double vt = v[p->target];
  if (vt > p->thr) p->depol = 1;
  if (p->depol && vt < p->thr) p->repol = 1;
  if (p->repol && !p->fired) {
    p->fired = 1;
    p->t_fire = t;
    if (p->kind == CEP_S2_RESET) p->reset_now = 1;
    if (p->kind == CEP_S2_ECTOPIC) p->ecto_on = 1;
  }
  if (p->kind == CEP_S2_ECTOPIC && p->fired && t - p->t_fire > p->dur) p->ecto_on = 0;
}

// S2: the region back to its snapshot, in the step the protocol fired.
__global__ void s2_reset_kernel(const CepProto *p, double *y, int64_t ld, int ns, const int *nodes, int count,
                                const double *snap) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= count || !p->reset_now) return;
  const int64_t i = nodes[k];
  for (int s = 0; s < ns; ++s) y[(int64_t)s * ld + i] = snap[(int64_t)s * count + k];
}

int tissue_pre_step(cep_tissue *t) {
  if (t->proto_kind == CEP_S2_NONE) return CEP_OK;
  proto_kernel<<<1, 1, 0, t->stream>>>(t->proto, cep_internal_batch_v(t->cells), t->t, t->bcl, t->n_pace);
  if (t->proto_kind == CEP_S2_RESET && t->s2_count > 0) {
    int n = 0, ns = 0;
    cep_batch_size(t->cells, &n, &ns);
    long ld = 0;
    void *dev = nullptr;
    int rc = cep_batch_device_states(t->cells, &dev, &ld);
    if (rc) return rc;
    s2_reset_kernel<<<(t->s2_count + 255) / 256, 256, 0, t->stream>>>(t->proto, static_cast<double *>(dev), ld,
                                                                       t->ns, t->s2_nodes, t->s2_count, t->s2_snap);
  }
  FEM_CUDA(cudaGetLastError());
  return CEP_OK;
}

}  // namespace

extern "C" {

int cep_fem_create_grid(int dim, int nx, int ny, int nz, double h, double dt, const double *D, int n_d, int format,
                        void *stream, cep_fem_t *out) {
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
  const int64_t n_elem = (int64_t)(nx - 1) * (ny - 1) * (dim == 3 ? nz - 1 : 1);
  for (int64_t e = 0; e < n_elem * n_d; ++e)
    if (!std::isfinite(D[e])) return fail_msg(CEP_ERR_ARG, "D[%lld] is not finite", (long long)e);
  cep_fem *f = new cep_fem;
  f->n = (int)n;
  f->ld = (n + 31) / 32 * 32;
  f->dt = dt;
  f->stream = (cudaStream_t)stream;
  f->width = dim == 2 ? 9 : 27;
  f->dim = dim; f->gnx = nx; f->gny = ny; f->gnz = nz;
  // row pointers: neighbours per axis are 1 + (i > 0) + (i < n-1)
  std::vector<int> rp(n + 1);
  int64_t p = 0;
  auto cnt = [](int i, int m) { return 1 + (i > 0) + (i < m - 1); };
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        rp[(size_t)i + (size_t)nx * ((size_t)j + (size_t)ny * k)] = (int)p;
        p += (int64_t)cnt(i, nx) * cnt(j, ny) * (dim == 3 ? cnt(k, nz) : 1);
      }
  rp[n] = (int)p;
  f->nnz = p;
  int rc;
  double *d_D = nullptr;
  if ((rc = fem_alloc(f, &f->rp, (size_t)n + 1)) || (rc = fem_alloc(f, &f->col, (size_t)p)) ||
      (rc = fem_alloc(f, &f->a, (size_t)p)) || (rc = fem_alloc(f, &f->b, (size_t)p)) ||
      (rc = fem_alloc(f, &f->ecol, (size_t)f->width * f->ld)) || (rc = fem_alloc(f, &f->ea, (size_t)f->width * f->ld)) ||
      (rc = fem_alloc(f, &f->eb, (size_t)f->width * f->ld)) || (rc = fem_alloc(f, &f->dinv, (size_t)f->ld)) ||
      (rc = fem_alloc(f, &f->sa, (size_t)f->width * f->ld)) || (rc = fem_alloc(f, &f->sb, (size_t)f->width * f->ld))) {
    fem_free(f);
    return rc;
  }
  if ((rc = fem_alloc(f, &d_D, (size_t)n_elem * n_d))) {
    fem_free(f);
    return rc;
  }
  f->D = d_D;
  f->n_d = n_d;
  f->h = h;
  cudaError_t e = cudaMemcpyAsync(f->rp, rp.data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice, f->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_D, D, sizeof(double) * n_elem * n_d, cudaMemcpyHostToDevice, f->stream);
  if (e == cudaSuccess && cep_internal_fem_assemble_grid(dim, nx, ny, nz, h, dt, d_D, n_d, f->rp, f->col, f->a, f->b,
                                                        f->width, f->ld, f->ecol, f->ea, f->eb, f->dinv, f->stream))
    e = cudaGetLastError();
  if (e == cudaSuccess) {
    csr_to_stencil_kernel<<<(unsigned)((n + 127) / 128), 128, 0, f->stream>>>(n, nx, ny, dim, f->rp, f->col, f->a, f->b,
                                                                            f->ld, f->sa, f->sb);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(f->stream);
  if (e != cudaSuccess) {
    fem_free(f);
    return fail_msg(CEP_ERR_CUDA, "grid assembly failed: %s", cudaGetErrorString(e));
  }
  if ((rc = fem_build_classes(f)) || (rc = fem_finish_setup(f)) || (rc = fem_set_format(f, format))) {
    fem_free(f);
    return rc;
  }
  *out = f;
  return CEP_OK;
}

int cep_fem_create_tet(int n_nodes, const double *xyz, int n_elem, const int *conn, const double *D, int n_d,
                       double dt, int format, void *stream, cep_fem_t *out) {
  if (!out || !xyz || !conn || !D) return fail_msg(CEP_ERR_ARG, "null argument");
  *out = nullptr;
  if (n_nodes < 4 || n_elem < 1) return fail_msg(CEP_ERR_ARG, "mesh needs >= 4 nodes and >= 1 element");
  if (n_d != 1 && n_d != 6) return fail_msg(CEP_ERR_ARG, "n_d must be 1 (scalar) or 6 (tensor)");
  if (!(dt > 0)) return fail_msg(CEP_ERR_ARG, "dt must be positive");
  if (format == CEP_FEM_STENCIL || format == CEP_FEM_CLASSED)
    return fail_msg(CEP_ERR_ARG, "grid formats need a structured grid");
  for (long k = 0; k < 4L * n_elem; ++k)
    if (conn[k] < 0 || conn[k] >= n_nodes) return fail_msg(CEP_ERR_ARG, "element node %d out of range", conn[k]);
  // node -> (element, local node) in ascending element order, and each row's
  // columns: the nodes sharing an element with it, ascending
  std::vector<int> inc_ptr(n_nodes + 1, 0), fill(n_nodes, 0);
  for (long k = 0; k < 4L * n_elem; ++k) inc_ptr[conn[k] + 1]++;
  for (int i = 0; i < n_nodes; ++i) inc_ptr[i + 1] += inc_ptr[i];
  std::vector<int> inc(2 * (size_t)inc_ptr[n_nodes]);
  for (int e = 0; e < n_elem; ++e)
    for (int k = 0; k < 4; ++k) {
      const int i = conn[4 * (size_t)e + k], p = inc_ptr[i] + fill[i]++;
      inc[2 * (size_t)p] = e;
      inc[2 * (size_t)p + 1] = k;
    }
  std::vector<int> rp(n_nodes + 1, 0), col, nb;
  for (int i = 0; i < n_nodes; ++i) {
    nb.clear();
    for (int p = inc_ptr[i]; p < inc_ptr[i + 1]; ++p)
      for (int k = 0; k < 4; ++k) nb.push_back(conn[4 * (size_t)inc[2 * (size_t)p] + k]);
    std::sort(nb.begin(), nb.end());
    nb.erase(std::unique(nb.begin(), nb.end()), nb.end());
    col.insert(col.end(), nb.begin(), nb.end());
    rp[i + 1] = (int)col.size();
  }
  const size_t nnz = col.size();
  cudaStream_t st = (cudaStream_t)stream;
  double *d_xyz = nullptr, *d_D = nullptr, *d_a = nullptr, *d_b = nullptr;
  int *d_conn = nullptr, *d_incp = nullptr, *d_inc = nullptr, *d_rp = nullptr, *d_col = nullptr;
  auto release = [&] {
    for (void *q : {(void *)d_xyz, (void *)d_D, (void *)d_a, (void *)d_b, (void *)d_conn, (void *)d_incp,
                    (void *)d_inc, (void *)d_rp, (void *)d_col})
      cudaFree(q);
  };
  bool ok = cudaMalloc(&d_xyz, sizeof(double) * 3 * (size_t)n_nodes) == cudaSuccess &&
            cudaMalloc(&d_D, sizeof(double) * (size_t)n_d * n_elem) == cudaSuccess &&
            cudaMalloc(&d_a, sizeof(double) * nnz) == cudaSuccess && cudaMalloc(&d_b, sizeof(double) * nnz) == cudaSuccess &&
            cudaMalloc(&d_conn, sizeof(int) * 4 * (size_t)n_elem) == cudaSuccess &&
            cudaMalloc(&d_incp, sizeof(int) * inc_ptr.size()) == cudaSuccess &&
            cudaMalloc(&d_inc, sizeof(int) * inc.size()) == cudaSuccess &&
            cudaMalloc(&d_rp, sizeof(int) * rp.size()) == cudaSuccess && cudaMalloc(&d_col, sizeof(int) * nnz) == cudaSuccess;
  if (!ok) {
    release();
    return fail_msg(CEP_ERR_OOM, "tetrahedral assembly buffers");
  }
  cudaError_t e = cudaMemcpyAsync(d_xyz, xyz, sizeof(double) * 3 * (size_t)n_nodes, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_D, D, sizeof(double) * (size_t)n_d * n_elem, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_conn, conn, sizeof(int) * 4 * (size_t)n_elem, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_incp, inc_ptr.data(), sizeof(int) * inc_ptr.size(), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_inc, inc.data(), sizeof(int) * inc.size(), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_rp, rp.data(), sizeof(int) * rp.size(), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_col, col.data(), sizeof(int) * nnz, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess && cep_internal_fem_assemble_tet(n_nodes, d_xyz, d_conn, d_D, n_d, dt, d_incp, d_inc, d_rp, d_col,
                                                        d_a, d_b, st))
    e = cudaGetLastError();
  std::vector<double> a(nnz), b(nnz);
  if (e == cudaSuccess) e = cudaMemcpyAsync(a.data(), d_a, sizeof(double) * nnz, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(b.data(), d_b, sizeof(double) * nnz, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  release();
  if (e != cudaSuccess) return fail_msg(CEP_ERR_CUDA, "tetrahedral assembly failed: %s", cudaGetErrorString(e));
  return cep_fem_create_csr(n_nodes, rp.data(), col.data(), a.data(), b.data(), dt, format, stream, out);
}

int cep_fem_create_csr(int n, const int *row_ptr, const int *col_idx, const double *a_val, const double *b_val,
                       double dt, int format, void *stream, cep_fem_t *out) {
  if (!out || !row_ptr || !col_idx || !a_val || !b_val) return fail_msg(CEP_ERR_ARG, "null argument");
  *out = nullptr;
  if (n <= 0 || !(dt > 0)) return fail_msg(CEP_ERR_ARG, "n and dt must be positive");
  if (row_ptr[0] != 0) return fail_msg(CEP_ERR_ARG, "row_ptr[0] must be 0");
  int width = 0;
  for (int i = 0; i < n; ++i) {
    if (row_ptr[i + 1] < row_ptr[i]) return fail_msg(CEP_ERR_ARG, "row_ptr is not monotone at row %d", i);
    width = std::max(width, row_ptr[i + 1] - row_ptr[i]);
  }
  const int64_t nnz = row_ptr[n];
  for (int64_t k = 0; k < nnz; ++k) {
    if (col_idx[k] < 0 || col_idx[k] >= n) return fail_msg(CEP_ERR_ARG, "col_idx[%lld] = %d out of range", (long long)k, col_idx[k]);
    if (!std::isfinite(a_val[k]) || !std::isfinite(b_val[k])) return fail_msg(CEP_ERR_ARG, "matrix entry %lld is not finite", (long long)k);
  }
  cep_fem *f = new cep_fem;
  f->n = n;
  f->ld = ((int64_t)n + 31) / 32 * 32;
  f->nnz = nnz;
  f->dt = dt;
  f->width = std::max(width, 1);
  f->stream = (cudaStream_t)stream;
  int rc;
  if ((rc = fem_alloc(f, &f->rp, (size_t)n + 1)) || (rc = fem_alloc(f, &f->col, (size_t)std::max<int64_t>(nnz, 1))) ||
      (rc = fem_alloc(f, &f->a, (size_t)std::max<int64_t>(nnz, 1))) || (rc = fem_alloc(f, &f->b, (size_t)std::max<int64_t>(nnz, 1))) ||
      (rc = fem_alloc(f, &f->ecol, (size_t)f->width * f->ld)) || (rc = fem_alloc(f, &f->ea, (size_t)f->width * f->ld)) ||
      (rc = fem_alloc(f, &f->eb, (size_t)f->width * f->ld)) || (rc = fem_alloc(f, &f->dinv, (size_t)f->ld))) {
    fem_free(f);
    return rc;
  }
  cudaError_t e = cudaMemcpyAsync(f->rp, row_ptr, sizeof(int) * (n + 1), cudaMemcpyHostToDevice, f->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(f->col, col_idx, sizeof(int) * nnz, cudaMemcpyHostToDevice, f->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(f->a, a_val, sizeof(double) * nnz, cudaMemcpyHostToDevice, f->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(f->b, b_val, sizeof(double) * nnz, cudaMemcpyHostToDevice, f->stream);
  if (e == cudaSuccess) {
    csr_to_ell_kernel<<<(n + 127) / 128, 128, 0, f->stream>>>(n, f->rp, f->col, f->a, f->b, f->width, f->ld, f->ecol,
                                                              f->ea, f->eb, f->dinv);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(f->stream);
  if (e != cudaSuccess) {
    fem_free(f);
    return fail_msg(CEP_ERR_CUDA, "CSR upload failed: %s", cudaGetErrorString(e));
  }
  if ((rc = fem_finish_setup(f)) || (rc = fem_set_format(f, format))) {
    fem_free(f);
    return rc;
  }
  *out = f;
  return CEP_OK;
}

int cep_fem_destroy(cep_fem_t f) {
  if (!f) return CEP_OK;
  cudaStreamSynchronize(f->stream);
  fem_free(f);
  return CEP_OK;
}

int cep_fem_info(cep_fem_t f, int *n, long *nnz, int *format, int *ell_width) {
  if (!f) return fail_msg(CEP_ERR_ARG, "null operator");
  if (n) *n = f->n;
  if (nnz) *nnz = (long)f->nnz;
  if (format) *format = f->format;
  if (ell_width) *ell_width = f->width;
  return CEP_OK;
}

int cep_fem_set_format(cep_fem_t f, int format) {
  if (!f) return fail_msg(CEP_ERR_ARG, "null operator");
  return fem_set_format(f, format);
}

int cep_fem_get_csr(cep_fem_t f, int *row_ptr, int *col_idx, double *a_val, double *b_val) {
  if (!f) return fail_msg(CEP_ERR_ARG, "null operator");
  if (row_ptr) FEM_CUDA(cudaMemcpyAsync(row_ptr, f->rp, sizeof(int) * (f->n + 1), cudaMemcpyDeviceToHost, f->stream));
  if (col_idx) FEM_CUDA(cudaMemcpyAsync(col_idx, f->col, sizeof(int) * f->nnz, cudaMemcpyDeviceToHost, f->stream));
  if (a_val) FEM_CUDA(cudaMemcpyAsync(a_val, f->a, sizeof(double) * f->nnz, cudaMemcpyDeviceToHost, f->stream));
  if (b_val) FEM_CUDA(cudaMemcpyAsync(b_val, f->b, sizeof(double) * f->nnz, cudaMemcpyDeviceToHost, f->stream));
  FEM_CUDA(cudaStreamSynchronize(f->stream));
  return CEP_OK;
}

int cep_fem_set_solver(cep_fem_t f, double rtol, int max_iter, int precond_norm) {
  if (!f) return fail_msg(CEP_ERR_ARG, "null operator");
  if (!(rtol > 0) || max_iter <= 0 || max_iter > CEP_FEM_MAX_ITER)
    return fail_msg(CEP_ERR_ARG, "rtol must be positive and max_iter in 1..%d", CEP_FEM_MAX_ITER);
  f->rtol = rtol;
  f->max_iter = max_iter;
  f->precond_norm = precond_norm ? 1 : 0;
  return CEP_OK;
}

int cep_fem_spmv(cep_fem_t f, int which, const double *x, double *y) {
  if (!f || !x || !y) return fail_msg(CEP_ERR_ARG, "null argument");
  double *dx = f->q, *dy = f->r;  // scratch vectors of the solver
  FEM_CUDA(cudaMemcpyAsync(dx, x, sizeof(double) * f->n, cudaMemcpyHostToDevice, f->stream));
  const unsigned grid = (unsigned)((f->n + 255) / 256);
  with_view(f, [&](auto m) {
    spmv_kernel<<<grid, 256, 0, f->stream>>>(m, which ? 1 : 0, (int64_t)f->n, dx, dy);
    return 0;
  });
  FEM_CUDA(cudaGetLastError());
  FEM_CUDA(cudaMemcpyAsync(y, dy, sizeof(double) * f->n, cudaMemcpyDeviceToHost, f->stream));
  FEM_CUDA(cudaStreamSynchronize(f->stream));
  return CEP_OK;
}

int cep_fem_solve_device(cep_fem_t f, void *d_v) {
  if (!f || !d_v) return fail_msg(CEP_ERR_ARG, "null argument");
  return fem_solve_async(f, (double *)d_v, nullptr, 0.0, 0.0);
}

int cep_fem_solve(cep_fem_t f, double *v, int *iters, double *rel_res) {
  if (!f || !v) return fail_msg(CEP_ERR_ARG, "null argument");
  double *dv = nullptr;
  FEM_CUDA(cudaMallocAsync((void **)&dv, sizeof(double) * f->n, f->stream));
  int rc = CEP_OK;
  cudaError_t e = cudaMemcpyAsync(dv, v, sizeof(double) * f->n, cudaMemcpyHostToDevice, f->stream);
  if (e == cudaSuccess) rc = fem_solve_async(f, dv, nullptr, 0.0, 0.0);
  if (e == cudaSuccess && rc == CEP_OK) e = cudaMemcpyAsync(v, dv, sizeof(double) * f->n, cudaMemcpyDeviceToHost, f->stream);
  cudaFreeAsync(dv, f->stream);
  if (e != cudaSuccess) return fail_msg(CEP_ERR_CUDA, "solve transfer failed: %s", cudaGetErrorString(e));
  if (rc) return rc;
  if ((rc = fem_check_ctl(f))) return rc;
  Status s;
  FEM_CUDA(copy_sync(&s, f->st, sizeof(Status), cudaMemcpyDeviceToHost, f->stream));
  if (iters) *iters = s.last_iters;
  if (rel_res) *rel_res = s.last_res;
  if (s.last_iters < 0) return fail_msg(CEP_ERR_NOT_CONVERGED, "PCG hit max_iter (%d), relative residual %g", f->max_iter, s.last_res);
  return CEP_OK;
}

int cep_fem_stats(cep_fem_t f, int *last_iters, long *total_iters, long *solves, int *not_converged, double *last_res) {
  if (!f) return fail_msg(CEP_ERR_ARG, "null operator");
  int rc;
  if ((rc = fem_check_ctl(f))) return rc;
  Status s;
  FEM_CUDA(copy_sync(&s, f->st, sizeof(Status), cudaMemcpyDeviceToHost, f->stream));
  if (last_iters) *last_iters = s.last_iters;
  if (total_iters) *total_iters = (long)s.total_iters;
  if (solves) *solves = (long)s.solves;
  if (not_converged) *not_converged = s.not_converged;
  if (last_res) *last_res = s.last_res;
  return CEP_OK;
}

}  // extern "C"

// --------------------------------------------------------- tissue groups
struct cep_tissue_group {
  std::vector<cep_tissue_t> ts;
  int format = 0, dim = 0, grid = 0;
  cudaStream_t stream = nullptr;
  std::vector<unsigned char> ops;  // PcgOps<View>, passed by value at each launch
  Ctl *ctl = nullptr;
  int *ops_done = nullptr;
  // optional per-phase timing: three events per step (before the ionic
  // launches, before the diffusion launch, after it), folded into the
  // totals when read or when the pool is used up
  bool timing = false;
  std::vector<cudaEvent_t> ev;
  size_t ev_used = 0;
  double ionic_ms = 0.0, diffusion_ms = 0.0;
  long timed_steps = 0;
};

namespace {

constexpr size_t kGroupEvents = 3 * 1024;

int group_fold_timing(cep_tissue_group *g) {
  if (g->ev_used == 0) return CEP_OK;
  FEM_CUDA(cudaEventSynchronize(g->ev[g->ev_used - 1]));
  for (size_t k = 0; k + 3 <= g->ev_used; k += 3) {
    float a = 0.f, b = 0.f;
    FEM_CUDA(cudaEventElapsedTime(&a, g->ev[k], g->ev[k + 1]));
    FEM_CUDA(cudaEventElapsedTime(&b, g->ev[k + 1], g->ev[k + 2]));
    g->ionic_ms += a;
    g->diffusion_ms += b;
    ++g->timed_steps;
  }
  g->ev_used = 0;
  return CEP_OK;
}

int group_event(cep_tissue_group *g) {
  if (g->ev_used == g->ev.size()) {
    cudaEvent_t e;
    FEM_CUDA(cudaEventCreate(&e));
    g->ev.push_back(e);
  }
  FEM_CUDA(cudaEventRecord(g->ev[g->ev_used++], g->stream));
  return CEP_OK;
}

template <class M>
int group_build(cep_tissue_group *g, const std::vector<int> &nb, M (*view)(const cep_fem *)) {
  std::vector<PcgOp<M>> h(g->ts.size());
  int b0 = 0;
  for (size_t k = 0; k < g->ts.size(); ++k) {
    cep_fem *f = g->ts[k]->fem;
    PcgOp<M> &o = h[k];
    o.m = view(f);
    o.a.n = f->n; o.a.ld = f->ld; o.a.dt = f->dt; o.a.rtol = f->rtol; o.a.max_iter = f->max_iter;
    o.a.precond_norm = f->precond_norm;
    o.a.v = cep_internal_batch_v(g->ts[k]->cells);
    o.a.dinv = f->dinv;
    o.a.r = f->r; o.a.q = f->q; o.a.p0 = f->p0; o.a.p1 = f->p1; o.a.z = f->z;
    o.a.part = f->part;
    o.a.ctl = nullptr;
    o.a.st = f->st;
    o.a.tact = g->ts[k]->tact;
    o.a.t_new = 0.0;
    o.a.act_thr = g->ts[k]->act_thr;
    o.block0 = b0;
    o.nblocks = nb[k];
    b0 += nb[k];
  }
  g->grid = b0;
  g->ops.assign(sizeof(PcgOps<M>), 0);
  std::memcpy(g->ops.data(), h.data(), sizeof(PcgOp<M>) * h.size());
  return CEP_OK;
}

// Each operator's activation time stamp is its own tissue's time after the
// step (tissues of a group may run at different times and dt).
template <class M>
int group_launch(cep_tissue_group *g) {
  int n = (int)g->ts.size();
  PcgOps<M> *ops = reinterpret_cast<PcgOps<M> *>(g->ops.data());
  for (int k = 0; k < n; ++k) ops->op[k].a.t_new = g->ts[k]->t + g->ts[k]->dt;
  Ctl *ctl = g->ctl;
  int *done = g->ops_done;
  void *args[] = {g->ops.data(), &n, &ctl, &done};
  FEM_CUDA(cudaMemsetAsync(g->ctl, 0, sizeof(Ctl) + 64, g->stream));
  FEM_CUDA(cudaLaunchCooperativeKernel((const void *)pcg_many_kernel<M>, dim3(g->grid), dim3(kPcgBlock), args, 0,
                                       g->stream));
  return CEP_OK;
}

}  // namespace

extern "C" {

int cep_tissue_group_create(const cep_tissue_t *ts, int count, cep_tissue_group_t *out) {
  if (!ts || !out || count <= 0) return fail_msg(CEP_ERR_ARG, "bad tissue list");
  *out = nullptr;
  int dev = 0, sms = 0;
  FEM_CUDA(cudaGetDevice(&dev));
  FEM_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  if (count > sms || count > kMaxGroup)
    return fail_msg(CEP_ERR_ARG, "at most %d tissues per group (one SM each at least)", std::min(sms, kMaxGroup));
  for (int k = 0; k < count; ++k) {
    if (!ts[k]) return fail_msg(CEP_ERR_ARG, "tissue %d is NULL", k);
    const cep_fem *f = ts[k]->fem, *f0 = ts[0]->fem;
    if (f->stream != f0->stream) return fail_msg(CEP_ERR_ARG, "tissues of a group share one stream");
    if (f->format != f0->format || f->dim != f0->dim)
      return fail_msg(CEP_ERR_ARG, "tissues of a group share one sparse format (and grid dimension)");
    for (int j = 0; j < k; ++j)
      if (ts[j] == ts[k]) return fail_msg(CEP_ERR_ARG, "tissue %d appears twice", k);
  }
  // blocks in proportion to rows, at least one each, at most the operator's
  // own partial slots, in total one per SM
  std::vector<int> nb(count);
  double total = 0;
  for (int k = 0; k < count; ++k) total += ts[k]->fem->n;
  int sum = 0;
  for (int k = 0; k < count; ++k) {
    nb[k] = std::max(1, std::min(ts[k]->fem->grid, (int)std::floor(sms * ts[k]->fem->n / total)));
    sum += nb[k];
  }
  while (sum > sms) {
    int kmax = (int)(std::max_element(nb.begin(), nb.end()) - nb.begin());
    nb[kmax] -= 1;
    sum -= 1;
  }
  cep_tissue_group *g = new cep_tissue_group;
  g->ts.assign(ts, ts + count);
  g->format = ts[0]->fem->format;
  g->dim = ts[0]->fem->dim;
  g->stream = ts[0]->fem->stream;
  if (cudaMalloc((void **)&g->ctl, sizeof(Ctl) + 64) != cudaSuccess) {
    delete g;
    return fail_msg(CEP_ERR_OOM, "group control words");
  }
  g->ops_done = reinterpret_cast<int *>(reinterpret_cast<char *>(g->ctl) + sizeof(Ctl));
  int rc;
  if (g->format == CEP_FEM_CSR)
    rc = group_build(g, nb, csr_view);
  else if (g->format == CEP_FEM_STENCIL)
    rc = g->dim == 3 ? group_build(g, nb, stencil_view<3>) : group_build(g, nb, stencil_view<2>);
  else if (g->format == CEP_FEM_CLASSED)
    rc = g->dim == 3 ? group_build(g, nb, class_view<3>) : group_build(g, nb, class_view<2>);
  else
    rc = group_build(g, nb, ell_view);
  if (rc) {
    cudaFree(g->ctl);
    delete g;
    return rc;
  }
  *out = g;
  return CEP_OK;
}

int cep_tissue_group_destroy(cep_tissue_group_t g) {
  if (!g) return CEP_OK;
  cudaStreamSynchronize(g->stream);
  for (cudaEvent_t e : g->ev) cudaEventDestroy(e);
  cudaFree(g->ctl);
  delete g;
  return CEP_OK;
}

int cep_tissue_group_set_timing(cep_tissue_group_t g, int on) {
  if (!g) return fail_msg(CEP_ERR_ARG, "null group");
  int rc;
  if ((rc = group_fold_timing(g))) return rc;
  g->timing = on != 0;
  g->ionic_ms = g->diffusion_ms = 0.0;
  g->timed_steps = 0;
  return CEP_OK;
}

int cep_tissue_group_timing(cep_tissue_group_t g, double *ionic_ms, double *diffusion_ms, long *steps) {
  if (!g) return fail_msg(CEP_ERR_ARG, "null group");
  int rc;
  if ((rc = group_fold_timing(g))) return rc;
  if (ionic_ms) *ionic_ms = g->ionic_ms;
  if (diffusion_ms) *diffusion_ms = g->diffusion_ms;
  if (steps) *steps = g->timed_steps;
  return CEP_OK;
}

int cep_tissue_group_run(cep_tissue_group_t g, long n_steps) {
  if (!g) return fail_msg(CEP_ERR_ARG, "null group");
  if (n_steps < 0) return fail_msg(CEP_ERR_ARG, "n_steps must be >= 0");
  for (long s = 0; s < n_steps; ++s) {
    int rc;
    if (g->timing) {
      if (g->ev_used + 3 > kGroupEvents && (rc = group_fold_timing(g))) return rc;
      if ((rc = group_event(g))) return rc;
    }
    for (cep_tissue_t t : g->ts) {
      if ((rc = tissue_pre_step(t))) return rc;
      rc = cep_internal_batch_tissue_step(t->cells, t->mask, t->t, t->bcl, t->t_crt, t->dur, t->n_pace, t->proto,
                                          t->mask2);
      if (rc) return rc;
    }
    if (g->timing && (rc = group_event(g))) return rc;
    if (g->format == CEP_FEM_CSR)
      rc = group_launch<CsrView>(g);
    else if (g->format == CEP_FEM_STENCIL)
      rc = g->dim == 3 ? group_launch<StencilView<3>>(g) : group_launch<StencilView<2>>(g);
    else if (g->format == CEP_FEM_CLASSED)
      rc = g->dim == 3 ? group_launch<ClassView<3>>(g) : group_launch<ClassView<2>>(g);
    else
      rc = group_launch<EllView>(g);
    if (rc) return rc;
    if (g->timing && (rc = group_event(g))) return rc;
    for (cep_tissue_t t : g->ts) {
      t->t += t->dt;
      ++t->steps;
      if ((rc = ecg_record(t))) return rc;
    }
  }
  return CEP_OK;
}

}  // extern "C"

// ---------------------------------------------------------------- tissue
extern "C" {
int cep_tissue_create(cep_batch_t cells, cep_fem_t fem, double dt, cep_tissue_t *out) {
  if (!cells || !fem || !out) return fail_msg(CEP_ERR_ARG, "null argument");
  *out = nullptr;
  int n = 0, ns = 0;
  int rc = cep_batch_size(cells, &n, &ns);
  if (rc) return rc;
  if (n != fem->n) return fail_msg(CEP_ERR_ARG, "batch has %d instances, operator has %d rows", n, fem->n);
  if (!(dt > 0) || std::fabs(dt - fem->dt) > 1e-12 * dt)
    return fail_msg(CEP_ERR_ARG, "dt %g differs from the operator's dt %g", dt, fem->dt);
  if ((cudaStream_t)cep_internal_batch_stream(cells) != fem->stream)
    return fail_msg(CEP_ERR_ARG, "batch and operator must share one stream");
  if ((rc = cep_internal_batch_tissue_begin(cells, dt))) return rc;
  cep_tissue *t = new cep_tissue;
  t->cells = cells;
  t->fem = fem;
  t->stream = fem->stream;
  t->n = n;
  t->dt = dt;
  if (cudaMalloc((void **)&t->mask, (size_t)n) != cudaSuccess || cudaMalloc((void **)&t->tact, sizeof(double) * n) != cudaSuccess) {
    cudaFree(t->mask);
    delete t;
    return fail_msg(CEP_ERR_OOM, "tissue buffers");
  }
  std::vector<double> neg(n, -1.0);
  cudaMemsetAsync(t->mask, 0, (size_t)n, t->stream);
  cudaMemcpyAsync(t->tact, neg.data(), sizeof(double) * n, cudaMemcpyHostToDevice, t->stream);
  if (cudaStreamSynchronize(t->stream) != cudaSuccess) {
    cudaFree(t->mask);
    cudaFree(t->tact);
    delete t;
    return fail_msg(CEP_ERR_CUDA, "tissue set-up failed");
  }
  *out = t;
  return CEP_OK;
}

int cep_tissue_destroy(cep_tissue_t t) {
  if (!t) return CEP_OK;
  cudaStreamSynchronize(t->stream);
  cudaFree(t->mask);
  cudaFree(t->tact);
  cudaFree(t->el);
  cudaFree(t->ecg_part);
  cudaFree(t->ecg_rec);
  cudaFree(t->proto);
  cudaFree(t->mask2);
  cudaFree(t->s2_nodes);
  cudaFree(t->s2_snap);
  delete t;
  return CEP_OK;
}

int cep_tissue_set_stimulus(cep_tissue_t t, const unsigned char *s1_mask, double bcl, double t_crt, double dur,
                            int n_pace) {
  if (!t || !s1_mask) return fail_msg(CEP_ERR_ARG, "null argument");
  if (!(bcl > 0) || !(dur >= 0) || n_pace < 0) return fail_msg(CEP_ERR_ARG, "bad stimulus protocol");
  FEM_CUDA(cudaMemcpyAsync(t->mask, s1_mask, (size_t)t->n, cudaMemcpyHostToDevice, t->stream));
  FEM_CUDA(cudaStreamSynchronize(t->stream));
  t->bcl = bcl;
  t->t_crt = t_crt;
  t->dur = dur;
  t->n_pace = n_pace;
  return CEP_OK;
}

int cep_tissue_set_activation_threshold(cep_tissue_t t, double vm_threshold) {
  if (!t) return fail_msg(CEP_ERR_ARG, "null argument");
  t->act_thr = vm_threshold;
  return CEP_OK;
}

int cep_tissue_set_clock(cep_tissue_t t, double time) {
  if (!t) return fail_msg(CEP_ERR_ARG, "null argument");
  if (!std::isfinite(time) || time < 0) return fail_msg(CEP_ERR_ARG, "time must be finite and >= 0");
  FEM_CUDA(cudaStreamSynchronize(t->stream));
  t->t = time;
  return CEP_OK;
}

int cep_tissue_run(cep_tissue_t t, long n_steps) {
  if (!t) return fail_msg(CEP_ERR_ARG, "null argument");
  if (n_steps < 0) return fail_msg(CEP_ERR_ARG, "n_steps must be >= 0");
  double *v = cep_internal_batch_v(t->cells);
  for (long s = 0; s < n_steps; ++s) {
    int rc = tissue_pre_step(t);
    if (rc) return rc;
    rc = cep_internal_batch_tissue_step(t->cells, t->mask, t->t, t->bcl, t->t_crt, t->dur, t->n_pace, t->proto,
                                        t->mask2);
    if (rc) return rc;
    t->t += t->dt;
    ++t->steps;
    if ((rc = fem_solve_async(t->fem, v, t->tact, t->t, t->act_thr))) return rc;
    if ((rc = ecg_record(t))) return rc;
  }
  return CEP_OK;
}

int cep_tissue_set_electrodes(cep_tissue_t t, int n_el, const double *xyz, long every, long max_records) {
  if (!t) return fail_msg(CEP_ERR_ARG, "null argument");
  if (n_el < 0 || (n_el > 0 && !xyz) || every <= 0 || max_records < 0)
    return fail_msg(CEP_ERR_ARG, "bad electrode set (n_el >= 0, every > 0, max_records >= 0)");
  if (n_el > 0 && !t->fem->D) return fail_msg(CEP_ERR_UNSUPPORTED, "pseudo-ECG needs a grid operator");
  FEM_CUDA(cudaStreamSynchronize(t->stream));
  cudaFree(t->el);
  cudaFree(t->ecg_part);
  cudaFree(t->ecg_rec);
  t->el = t->ecg_part = t->ecg_rec = nullptr;
  t->n_el = 0;
  t->ecg_n = 0;
  if (n_el == 0) return CEP_OK;
  const int blocks = ecg_blocks();
  if (cudaMalloc((void **)&t->el, sizeof(double) * 3 * n_el) != cudaSuccess ||
      cudaMalloc((void **)&t->ecg_part, sizeof(double) * (size_t)n_el * blocks) != cudaSuccess ||
      cudaMalloc((void **)&t->ecg_rec, sizeof(double) * (size_t)n_el * std::max(1L, max_records)) != cudaSuccess) {
    cudaFree(t->el);
    cudaFree(t->ecg_part);
    cudaFree(t->ecg_rec);
    t->el = t->ecg_part = t->ecg_rec = nullptr;
    return fail_msg(CEP_ERR_OOM, "pseudo-ECG buffers");
  }
  FEM_CUDA(copy_sync(t->el, xyz, sizeof(double) * 3 * n_el, cudaMemcpyHostToDevice, t->stream));
  t->n_el = n_el;
  t->ecg_every = every;
  t->ecg_max = max_records;
  return CEP_OK;
}

int cep_tissue_set_s2(cep_tissue_t t, int kind, int target_node, double vm_threshold, const unsigned char *region,
                      double ectopic_dur) {
  if (!t) return fail_msg(CEP_ERR_ARG, "null argument");
  if (kind != CEP_S2_NONE && kind != CEP_S2_RESET && kind != CEP_S2_ECTOPIC)
    return fail_msg(CEP_ERR_ARG, "unknown protocol %d", kind);
  if (kind != CEP_S2_NONE && (!region || target_node < 0 || target_node >= t->n || !std::isfinite(vm_threshold)))
    return fail_msg(CEP_ERR_ARG, "protocol needs a region and a target node in 0..%d", t->n - 1);
  if (kind == CEP_S2_ECTOPIC && !(ectopic_dur >= 0)) return fail_msg(CEP_ERR_ARG, "ectopic_dur must be >= 0");
  FEM_CUDA(cudaStreamSynchronize(t->stream));
  cudaFree(t->proto);
  cudaFree(t->mask2);
  cudaFree(t->s2_nodes);
  cudaFree(t->s2_snap);
  t->proto = nullptr;
  t->mask2 = nullptr;
  t->s2_nodes = nullptr;
  t->s2_snap = nullptr;
  t->s2_count = 0;
  t->proto_kind = CEP_S2_NONE;
  if (kind == CEP_S2_NONE) return CEP_OK;
  CepProto p{};
  p.kind = kind;
  p.target = target_node;
  p.thr = vm_threshold;
  p.dur = ectopic_dur;
  std::vector<int> nodes;
  for (int i = 0; i < t->n; ++i)
    if (region[i]) nodes.push_back(i);
  int n = 0, ns = 0;
  int rc;
  if ((rc = cep_batch_size(t->cells, &n, &ns))) return rc;
  bool ok = cudaMalloc((void **)&t->proto, sizeof(CepProto)) == cudaSuccess;
  if (ok && kind == CEP_S2_ECTOPIC) {
    ok = cudaMalloc((void **)&t->mask2, (size_t)t->n) == cudaSuccess &&
         copy_sync(t->mask2, region, (size_t)t->n, cudaMemcpyHostToDevice, t->stream) == cudaSuccess;
  }
  if (ok && kind == CEP_S2_RESET && !nodes.empty()) {
    // snapshot of the region's states now (the batch's SoA rows)
    std::vector<double> all((size_t)ns * n), snap((size_t)ns * nodes.size());
    if ((rc = cep_batch_get_states(t->cells, all.data(), CEP_LAYOUT_SOA))) return rc;
    for (int s = 0; s < ns; ++s)
      for (size_t k = 0; k < nodes.size(); ++k) snap[(size_t)s * nodes.size() + k] = all[(size_t)s * n + nodes[k]];
    ok = cudaMalloc((void **)&t->s2_nodes, sizeof(int) * nodes.size()) == cudaSuccess &&
         cudaMalloc((void **)&t->s2_snap, sizeof(double) * snap.size()) == cudaSuccess &&
         copy_sync(t->s2_nodes, nodes.data(), sizeof(int) * nodes.size(), cudaMemcpyHostToDevice, t->stream) == cudaSuccess &&
         copy_sync(t->s2_snap, snap.data(), sizeof(double) * snap.size(), cudaMemcpyHostToDevice, t->stream) == cudaSuccess;
    t->s2_count = (int)nodes.size();
    t->ns = ns;
  }
  if (!ok || copy_sync(t->proto, &p, sizeof(CepProto), cudaMemcpyHostToDevice, t->stream) != cudaSuccess) {
    cudaFree(t->proto);
    cudaFree(t->mask2);
    cudaFree(t->s2_nodes);
    cudaFree(t->s2_snap);
    t->proto = nullptr;
    t->mask2 = nullptr;
    t->s2_nodes = nullptr;
    t->s2_snap = nullptr;
    t->s2_count = 0;
    return fail_msg(CEP_ERR_OOM, "S2 protocol buffers");
  }
  t->proto_kind = kind;
  return CEP_OK;
}

int cep_tissue_get_ecg(cep_tissue_t t, double *phi, long *n_records) {
  if (!t) return fail_msg(CEP_ERR_ARG, "null argument");
  FEM_CUDA(cudaStreamSynchronize(t->stream));
  if (n_records) *n_records = t->ecg_n;
  if (phi && t->ecg_n > 0)
    FEM_CUDA(copy_sync(phi, t->ecg_rec, sizeof(double) * (size_t)t->ecg_n * t->n_el, cudaMemcpyDeviceToHost, t->stream));
  return CEP_OK;
}

int cep_tissue_sync(cep_tissue_t t) {
  if (!t) return fail_msg(CEP_ERR_ARG, "null argument");
  FEM_CUDA(cudaStreamSynchronize(t->stream));
  return fem_check_ctl(t->fem);
}

int cep_tissue_get_v(cep_tissue_t t, double *v) {
  if (!t || !v) return fail_msg(CEP_ERR_ARG, "null argument");
  FEM_CUDA(cudaMemcpyAsync(v, cep_internal_batch_v(t->cells), sizeof(double) * t->n, cudaMemcpyDeviceToHost, t->stream));
  FEM_CUDA(cudaStreamSynchronize(t->stream));
  return CEP_OK;
}

int cep_tissue_get_activation(cep_tissue_t t, double *t_act) {
  if (!t || !t_act) return fail_msg(CEP_ERR_ARG, "null argument");
  FEM_CUDA(cudaMemcpyAsync(t_act, t->tact, sizeof(double) * t->n, cudaMemcpyDeviceToHost, t->stream));
  FEM_CUDA(cudaStreamSynchronize(t->stream));
  return CEP_OK;
}

int cep_tissue_stats(cep_tissue_t t, double *time, long *steps, long *cg_iters, int *not_converged) {
  if (!t) return fail_msg(CEP_ERR_ARG, "null argument");
  int rc = cep_tissue_sync(t);
  if (rc) return rc;
  long total = 0;
  int nc = 0;
  if ((rc = cep_fem_stats(t->fem, nullptr, &total, nullptr, &nc, nullptr))) return rc;
  if (time) *time = t->t;
  if (steps) *steps = t->steps;
  if (cg_iters) *cg_iters = total;
  if (not_converged) *not_converged = nc;
  return CEP_OK;
}

}  // extern "C"

// Test hook of the bounded barrier waits (no counterpart in the reference).
extern "C" int cep_fem_set_wait_test(long spin_limit, unsigned block0_delay_ns) {
  if (spin_limit < 0) return fail_msg(CEP_ERR_ARG, "spin_limit must be >= 0");
  if (block0_delay_ns > 100000000u) return fail_msg(CEP_ERR_ARG, "block0_delay_ns above 0.1 s");
  const long long lim = spin_limit;
  FEM_CUDA(cudaMemcpyToSymbol(cep::fem::g_spin_limit_test, &lim, sizeof(lim)));
  FEM_CUDA(cudaMemcpyToSymbol(cep::fem::g_block0_delay_ns, &block0_delay_ns, sizeof(block0_delay_ns)));
  FEM_CUDA(cudaDeviceSynchronize());  // landed before any stream's next launch reads them
  return CEP_OK;
}

// ------------------------------------------------------ allocation-free solve
// Jacobi-PCG on a caller-owned device CSR operator with the solver's work
// vectors in a fixed scratch area of this library (no counterpart in the
// reference). The scratch is one file-scope device array; its address is
// resolved once per device (the first call, which must precede any stream
// capture) and every later call only launches work. The cached address
// assumes the device's primary context lives as long as the process: after
// cudaDeviceReset the module is loaded again and the cache is stale. Calls
// that overlap in time on one device share the scratch and race: the caller
// serialises them.
namespace {

constexpr int64_t kNaRows = CEP_NOALLOC_MAX_ROWS;
constexpr int kNaMaxGrid = 1024;
// dinv, r, q, p0, p1, z | partials [3][kNaMaxGrid] | Ctl | Status | first bad row
constexpr int64_t kNaVecWords = 6 * kNaRows;
constexpr int64_t kNaWords = kNaVecWords + 3 * kNaMaxGrid + 8 + 8 + 8;

static __device__ __align__(256) double g_noalloc_scratch[kNaWords];

struct NaDevice {
  double *base = nullptr;
  int grid = 0;
};
NaDevice g_na_dev[64];
std::mutex g_na_mu;

// Jacobi inverse of the caller's operator. A row without a diagonal entry,
// or with a zero or non-finite one, keeps dinv = 1 so the solve stays finite,
// and its index goes to *bad (smallest such row) for the blocking form to
// report.
__global__ void noalloc_dinv_kernel(int64_t n, const int *rp, const int *col, const double *a, double *dinv,
                                    int *bad) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double diag = 0.0;
  for (int k = rp[i]; k < rp[i + 1]; ++k)
    if (col[k] == i) diag = a[k];
  if (diag == 0.0 || !isfinite(diag)) {
    atomicMin(bad, (int)i);
    diag = 1.0;
  }
  dinv[i] = 1.0 / diag;
}

}  // namespace

extern "C" int cep_fem_solve_csr_noalloc(int n, const void *d_row_ptr, const void *d_col_idx, const void *d_a_val,
                                         const void *d_b_val, double dt, double rtol, int max_iter, void *d_v,
                                         void *stream, int *iters_out) {
  if (!d_row_ptr || !d_col_idx || !d_a_val || !d_b_val || !d_v) return fail_msg(CEP_ERR_ARG, "null argument");
  if (n <= 0 || n > CEP_NOALLOC_MAX_ROWS)
    return fail_msg(CEP_ERR_ARG, "n = %d outside 1..%d (CEP_NOALLOC_MAX_ROWS)", n, CEP_NOALLOC_MAX_ROWS);
  if (!(dt > 0) || !(rtol > 0) || max_iter <= 0 || max_iter > CEP_FEM_MAX_ITER)
    return fail_msg(CEP_ERR_ARG, "dt and rtol must be positive and max_iter in 1..%d", CEP_FEM_MAX_ITER);
  int dev = 0;
  FEM_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return fail_msg(CEP_ERR_ARG, "device %d out of range", dev);
  NaDevice nd;
  {
    std::lock_guard<std::mutex> lock(g_na_mu);
    if (!g_na_dev[dev].base) {  // set-up: once per device
      void *p = nullptr;
      FEM_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
      int sms = 0, per_sm = 0;
      FEM_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
      FEM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pcg_kernel<CsrView>, kPcgBlock, 0));
      if (per_sm < 1) return fail_msg(CEP_ERR_CUDA, "PCG kernel does not fit on an SM");
      g_na_dev[dev].grid = std::min(sms, kNaMaxGrid);
      g_na_dev[dev].base = static_cast<double *>(p);
    }
    nd = g_na_dev[dev];
  }
  cudaStream_t st = (cudaStream_t)stream;
  double *base = nd.base;
  double *dinv = base, *r = base + kNaRows, *q = base + 2 * kNaRows, *part = base + kNaVecWords;
  double *p0 = base + 3 * kNaRows, *p1 = base + 4 * kNaRows, *z = base + 5 * kNaRows;
  Ctl *ctl = reinterpret_cast<Ctl *>(part + 3 * kNaMaxGrid);
  Status *stat = reinterpret_cast<Status *>(part + 3 * kNaMaxGrid + 8);
  int *bad = reinterpret_cast<int *>(part + 3 * kNaMaxGrid + 16);
  // the same grid rule as an operator handle: one block per SM, no more
  // blocks than rows need
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(nd.grid, (n + kPcgBlock - 1) / kPcgBlock));
  // what must start at zero: the barrier words and the counters
  FEM_CUDA(cudaMemsetAsync(ctl, 0, sizeof(Ctl), st));
  FEM_CUDA(cudaMemsetAsync(stat, 0, sizeof(Status), st));
  FEM_CUDA(cudaMemsetAsync(bad, 0x7f, sizeof(int), st));  // 0x7f7f7f7f: no bad row
  const CsrView m{static_cast<const int *>(d_row_ptr), static_cast<const int *>(d_col_idx),
                  static_cast<const double *>(d_a_val), static_cast<const double *>(d_b_val)};
  noalloc_dinv_kernel<<<(n + 127) / 128, 128, 0, st>>>(n, m.rp, m.col, m.a, dinv, bad);
  FEM_CUDA(cudaGetLastError());
  PcgArgs a;
  a.n = n;
  a.ld = n;
  a.dt = dt;
  a.rtol = rtol;
  a.max_iter = max_iter;
  a.precond_norm = 1;
  a.v = static_cast<double *>(d_v);
  a.dinv = dinv;
  a.r = r; a.q = q; a.p0 = p0; a.p1 = p1; a.z = z;
  a.part = part;
  a.ctl = ctl;
  a.st = stat;
  a.tact = nullptr;
  a.t_new = 0.0;
  a.act_thr = 0.0;
  CsrView mm = m;
  void *args[] = {&mm, &a};
  FEM_CUDA(cudaLaunchCooperativeKernel((const void *)pcg_kernel<CsrView>, dim3(grid), dim3(kPcgBlock), args, 0, st));
  if (iters_out) {  // blocking status read
    Ctl c;
    Status s;
    int first_bad = 0;
    FEM_CUDA(cudaMemcpyAsync(&c, ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, st));
    FEM_CUDA(cudaMemcpyAsync(&s, stat, sizeof(Status), cudaMemcpyDeviceToHost, st));
    FEM_CUDA(cudaMemcpyAsync(&first_bad, bad, sizeof(int), cudaMemcpyDeviceToHost, st));
    FEM_CUDA(cudaStreamSynchronize(st));
    if (first_bad != 0x7f7f7f7f)
      return fail_msg(CEP_ERR_ARG, "row %d has no usable diagonal entry (missing, zero or not finite)", first_bad);
    if (c.err) return fail_msg(CEP_ERR_TIMEOUT, "PCG grid barrier ran out of its spin limit");
    *iters_out = s.last_iters;
    if (s.last_iters < 0) return fail_msg(CEP_ERR_NOT_CONVERGED, "PCG hit max_iter (%d)", max_iter);
  }
  return CEP_OK;
}
