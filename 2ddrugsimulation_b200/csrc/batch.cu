// Batched ionic-model runtime: device memory layout, the init / run / rates
// kernels for every model and precision, and the cep_batch_* C ABI
// (include/cep_b200.h).
//
// HBM layout of a batch of n instances (ld = n rounded up to 32 so every
// row starts on a 256-byte boundary and a warp's accesses coalesce):
//   states  [n_states][ld] f64   SoA, the reference STATES order
//   params  [n_params][ld] f64   per-instance constants (Hill-scaled)
//   clock   t[ld] f64, iout[ld] i32, status[ld] i32
//   sched   [4][ld] i32          imax, steps_per_bcl, print_freq, first_pace
//   bm      [kNumF][ld] f64, [kNumI][ld] i32   biomarker state machine
//   ca ring [cap][ld] f64 x2     cai samples of the current beat
// A launch keeps one instance per thread with its whole state in registers
// for n_steps steps; HBM is touched once per launch.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <type_traits>
#include <string>
#include <vector>

#include "../../include/cep_b200.h"
#include "biomarkers.cuh"
#include "cep_device.cuh"
#include "model_ord.cuh"
#include "model_tt2006.cuh"
#include "model_tt2004.cuh"
#include "model_tomek.cuh"
#include "hrv.cuh"
#include "internal.h"

namespace {

thread_local std::string g_last_error;

int fail(int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

#define CEP_CUDA(call)                                                                      \
  do {                                                                                      \
    cudaError_t e_ = (call);                                                                \
    if (e_ != cudaSuccess) return fail(CEP_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
  } while (0)

constexpr int kBlock = 128;

// A copy on the batch's own stream, finished before returning. A plain
// cudaMemcpy runs on the legacy stream, which a non-blocking stream does
// not wait for (a read-back can see a kernel's output half written), and
// returns before a pageable upload has landed.
int copy_sync(void *dst, const void *src, size_t bytes, cudaMemcpyKind kind, cudaStream_t s) {
  cudaError_t e = cudaMemcpyAsync(dst, src, bytes, kind, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  return e == cudaSuccess ? CEP_OK : fail(CEP_ERR_CUDA, "copy of %zu bytes: %s", bytes, cudaGetErrorString(e));
}

}  // namespace

struct cep_batch {
  int model = 0, n = 0, ns = 0, np = 0, precision = 0;
  int64_t ld = 0;
  cudaStream_t stream = nullptr;
  double *states = nullptr, *params = nullptr, *t = nullptr;
  int *iout = nullptr, *status = nullptr, *sched = nullptr;
  double *bmf = nullptr, *ca_t = nullptr, *ca_v = nullptr;
  int *bmi = nullptr;
  int ca_cap = 0;
  bool initialized = false, has_protocol = false;
  double dt = 0.005, dt_write = 1.0, qnet_thr = -1e300;
  int n_pace = 0, first_pace = -1;
  int block = 128;    // threads per block of the one-thread-per-cell kernel
  int variant = CEP_KERNEL_CELL;  // CEP_KERNEL_*: cell, roles (4 warps / 32 cells), pairs (2 warps)
  std::vector<void *> allocs;
};

namespace cep {

// ------------------------------------------------------------------ traits
struct OrdModel {
  static constexpr bool kCipa = false;
  static constexpr bool kHasRates = true;  // the step runs under F64Rates
  static constexpr int kStates = ord::kNumStates;
  static constexpr int kParams = ord::kNumParams;
  static constexpr int kCai = ord::cai;
  template <class G> using Y = ord::Y<G>;
  template <class G> using Par = ord::Par<G>;
  template <class G> using Cur = ord::Cur<G>;
  template <class G>
  __device__ static void load(Y<G> &y, const double *s, int64_t ld, int64_t i) { ord::load(y, s, ld, i); }
  template <class G>
  __device__ static void store(const Y<G> &y, double *s, int64_t ld, int64_t i) { ord::store(y, s, ld, i); }
  template <class G>
  __device__ static void load_par(Par<G> &q, const double *p, int64_t ld, int64_t i) { ord::load_par(q, p, ld, i); }
  template <class P>
  __device__ static void step(Y<typename P::G> &y, const Par<typename P::G> &q, double t, double dt,
                              int stim_mode, bool update, Cur<typename P::G> &c) {
    ord::step<P>(y, q, t, dt, stim_mode, update, c);
  }
  __device__ static void init(double *par, double *s, int64_t ld, int64_t i, double ct, double conc,
                              const double *hill, unsigned flags) {
    ord::init_instance(par, s, ld, i, ct, conc, hill, flags & CEP_FLAG_DUTTA, flags & CEP_FLAG_QUIRKS,
                       flags & CEP_FLAG_NEO_ORD);
  }
  template <class G>
  __device__ static double cai_of(const Y<G> &y) { return y.cai; }
  __host__ __device__ static constexpr int p_bcl() { return ord::P_BCL; }
  __host__ __device__ static constexpr int p_stim_start() { return ord::P_stim_start; }
  __host__ __device__ static constexpr int p_duration() { return ord::P_duration; }
  __host__ __device__ static constexpr int p_amp() { return ord::P_amp; }
};

struct CipaModel : OrdModel {
  static constexpr bool kCipa = true;
  static constexpr int kStates = ord::cipa::kNumStates;
  static constexpr int kCai = ord::cipa::cai;
  template <class G>
  __device__ static void load(Y<G> &y, const double *s, int64_t ld, int64_t i) { ord::load_cipa(y, s, ld, i); }
  template <class G>
  __device__ static void store(const Y<G> &y, double *s, int64_t ld, int64_t i) { ord::store_cipa(y, s, ld, i); }
  template <class P>
  __device__ static void step(Y<typename P::G> &y, const Par<typename P::G> &q, double t, double dt,
                              int stim_mode, bool update, Cur<typename P::G> &c) {
    ord::step<P, true>(y, q, t, dt, stim_mode, update, c);
  }
  __device__ static void init(double *par, double *s, int64_t ld, int64_t i, double ct, double conc,
                              const double *hill, unsigned flags) {
    ord::init_instance_cipa(par, s, ld, i, ct, conc, hill, flags & CEP_FLAG_QUIRKS);
  }
};

struct Tt06Model {
  static constexpr bool kCipa = false;
  static constexpr bool kHasRates = false;
  static constexpr int kStates = tt06::kNumStates;
  static constexpr int kParams = tt06::kNumParams;
  static constexpr int kCai = tt06::Ca_i;
  template <class G> using Y = tt06::Y<G>;
  template <class G> using Par = tt06::Par<G>;
  template <class G> using Cur = tt06::Cur<G>;
  template <class G>
  __device__ static void load(Y<G> &y, const double *s, int64_t ld, int64_t i) { tt06::load(y, s, ld, i); }
  template <class G>
  __device__ static void store(const Y<G> &y, double *s, int64_t ld, int64_t i) { tt06::store(y, s, ld, i); }
  template <class G>
  __device__ static void load_par(Par<G> &q, const double *p, int64_t ld, int64_t i) { tt06::load_par(q, p, ld, i); }
  template <class P>
  __device__ static void step(Y<typename P::G> &y, const Par<typename P::G> &q, double t, double dt,
                              int stim_mode, bool update, Cur<typename P::G> &c) {
    tt06::step<P>(y, q, t, dt, stim_mode, update, c);
  }
  __device__ static void init(double *par, double *s, int64_t ld, int64_t i, double ct, double conc,
                              const double *hill, unsigned flags) {
    (void)ct; (void)flags;
    tt06::init_instance(par, s, ld, i, conc, hill);
  }
  template <class G>
  __device__ static double cai_of(const Y<G> &y) { return y.Ca_i; }
  __host__ __device__ static constexpr int p_bcl() { return tt06::P_BCL; }
  __host__ __device__ static constexpr int p_stim_start() { return tt06::P_stim_start; }
  __host__ __device__ static constexpr int p_duration() { return tt06::P_duration; }
  __host__ __device__ static constexpr int p_amp() { return tt06::P_amp; }
};

struct Tt04Model {
  static constexpr bool kCipa = false;
  static constexpr bool kHasRates = false;
  static constexpr int kStates = tt04::kNumStates;
  static constexpr int kParams = tt04::kNumParams;
  static constexpr int kCai = tt04::Ca_i;
  template <class G> using Y = tt04::Y<G>;
  template <class G> using Par = tt04::Par<G>;
  template <class G> using Cur = tt04::Cur<G>;
  template <class G>
  __device__ static void load(Y<G> &y, const double *s, int64_t ld, int64_t i) { tt04::load(y, s, ld, i); }
  template <class G>
  __device__ static void store(const Y<G> &y, double *s, int64_t ld, int64_t i) { tt04::store(y, s, ld, i); }
  template <class G>
  __device__ static void load_par(Par<G> &q, const double *p, int64_t ld, int64_t i) { tt04::load_par(q, p, ld, i); }
  template <class P>
  __device__ static void step(Y<typename P::G> &y, const Par<typename P::G> &q, double t, double dt,
                              int stim_mode, bool update, Cur<typename P::G> &c) {
    tt04::step<P>(y, q, t, dt, stim_mode, update, c);
  }
  __device__ static void init(double *par, double *s, int64_t ld, int64_t i, double ct, double conc,
                              const double *hill, unsigned flags) {
    (void)ct;
    tt04::init_instance(par, s, ld, i, conc, hill, (flags & CEP_FLAG_QUIRKS) != 0,
                        (flags & CEP_FLAG_TT04_MCELL) != 0);
  }
  template <class G>
  __device__ static double cai_of(const Y<G> &y) { return y.Ca_i; }
  __host__ __device__ static constexpr int p_bcl() { return tt04::P_BCL; }
  __host__ __device__ static constexpr int p_stim_start() { return tt04::P_stim_start; }
  __host__ __device__ static constexpr int p_duration() { return tt04::P_duration; }
  __host__ __device__ static constexpr int p_amp() { return tt04::P_amp; }
};

struct TomekModel {
  static constexpr bool kCipa = false;
  static constexpr bool kHasRates = true;
  static constexpr int kStates = tomek::kNumStates;
  static constexpr int kParams = tomek::kNumParams;
  static constexpr int kCai = tomek::cai;
  template <class G> using Y = tomek::Y<G>;
  template <class G> using Par = tomek::Par<G>;
  template <class G> using Cur = tomek::Cur<G>;
  template <class G>
  __device__ static void load(Y<G> &y, const double *s, int64_t ld, int64_t i) { tomek::load(y, s, ld, i); }
  template <class G>
  __device__ static void store(const Y<G> &y, double *s, int64_t ld, int64_t i) { tomek::store(y, s, ld, i); }
  template <class G>
  __device__ static void load_par(Par<G> &q, const double *p, int64_t ld, int64_t i) { tomek::load_par(q, p, ld, i); }
  template <class P>
  __device__ static void step(Y<typename P::G> &y, const Par<typename P::G> &q, double t, double dt,
                              int stim_mode, bool update, Cur<typename P::G> &c) {
    tomek::step<P>(y, q, t, dt, stim_mode, update, c);
  }
  __device__ static void init(double *par, double *s, int64_t ld, int64_t i, double ct, double conc,
                              const double *hill, unsigned flags) {
    tomek::init_instance(par, s, ld, i, ct, conc, hill, (flags & CEP_FLAG_QUIRKS) != 0);
  }
  template <class G>
  __device__ static double cai_of(const Y<G> &y) { return y.cai; }
  __host__ __device__ static constexpr int p_bcl() { return tomek::P_BCL; }
  __host__ __device__ static constexpr int p_stim_start() { return tomek::P_stim_start; }
  __host__ __device__ static constexpr int p_duration() { return tomek::P_duration; }
  __host__ __device__ static constexpr int p_amp() { return tomek::P_amp; }
};

// ----------------------------------------------------------------- kernels
// Instance ranges: every set-up kernel works on [first, first + count);
// the per-range inputs (celltype, conc, hill rows) are indexed from 0.
template <class M>
__global__ void init_kernel(double *par, double *s, int64_t ld, int64_t first, int count, const double *celltype,
                            const double *conc, const double *hill, int hill_stride, unsigned flags) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= count) return;
  const int64_t i = first + k;
  M::init(par, s, ld, i, celltype ? celltype[k] : 0.0, conc ? conc[k] : 0.0,
          hill ? hill + k * hill_stride : nullptr, flags);
}

__global__ void pacing_kernel(double *par, int64_t ld, int64_t first, int count, int p_bcl, int p_start, int p_dur,
                              int p_amp, double bcl, double start, double dur, double amp_scale) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= count) return;
  const int64_t i = first + k;
  par[p_bcl * ld + i] = bcl;
  if (start >= 0) par[p_start * ld + i] = start;
  if (dur >= 0) par[p_dur * ld + i] = dur;
  par[p_amp * ld + i] *= amp_scale;
}

// par[pidx][i] *= factor[i] for every instance (a caller's conductance
// scale, applied after init)
__global__ void scale_kernel(double *par, int64_t ld, int n, int pidx, const double *factor) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  par[pidx * ld + i] *= factor[i];
}

struct RunArgs {
  double *y;
  const double *par;
  int64_t ld;
  int n;
  double *t;
  int *iout;
  int *status;
  const int *sched;  // [4][ld]
  double dt;
  int n_steps;
  int bm_on;
  bm::View bv;
  double qnet_thr;
  int stim_mode;  // -1 periodic; 0/1 fixed tissue flag
};

__global__ void reset_kernel(RunArgs a, int64_t first, int count, int p_bcl, int p_start, int cai_idx) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= count) return;
  const int64_t i = first + k;
  a.t[i] = 0.0;
  a.iout[i] = 0;
  a.status[i] = CEP_INST_RUNNING;
  if (a.bm_on)
    bm::reset(a.bv, i, a.y[i], a.y[cai_idx * a.ld + i], a.par[p_bcl * a.ld + i], a.par[p_start * a.ld + i],
              a.dt);
}

// K fixed steps per instance with the biomarker state machine fused. One
// thread per instance; state, parameters and counters live in registers.
template <class M, class P>
__global__ void __launch_bounds__(kBlock) run_kernel(RunArgs a) {
  using G = typename P::G;
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  int st = a.status[i];
  if (st != CEP_INST_RUNNING) return;
  typename M::template Y<G> y;
  typename M::template Par<G> q;
  M::template load<G>(y, a.y, a.ld, i);
  M::template load_par<G>(q, a.par, a.ld, i);
  double t = a.t[i];
  int iout = a.iout[i];
  const bm::Sched sc{a.sched[i], a.sched[a.ld + i], a.sched[2 * a.ld + i], a.sched[3 * a.ld + i]};
  const bool bm_on = a.bm_on && sc.first_pace >= 0;
  int cnt_print = bm::countdown(iout, sc.print_freq);
  int cnt_bcl = bm::countdown(iout, sc.steps_per_bcl);
  const double bcl = a.par[M::p_bcl() * a.ld + i];
  const double stim_start = a.par[M::p_stim_start() * a.ld + i];
  typename M::template Cur<G> c;
  bm::Hot hot;
  if (bm_on) bm::hot_load(a.bv, i, hot);
  for (int k = 0; k <= a.n_steps; ++k) {
    const bool can_update = iout < sc.imax;
    if (can_update && k == a.n_steps) break;  // budget spent; sample iout is taken next launch
    const double V0 = y.V;
    const double cai0 = M::cai_of(y);
    M::template step<P>(y, q, t, a.dt, a.stim_mode, can_update, c);
    if (bm_on && iout >= 1)
      bm::sample(a.bv, i, sc, iout, t, a.dt, bcl, stim_start, V0, cai0, (double)c.dVdt, (double)c.INaL,
                 (double)c.ICaL, (double)c.Ito, (double)c.IKr, (double)c.IKs, (double)c.IK1, a.qnet_thr,
                 cnt_print, cnt_bcl, hot);
    if (!can_update) {
      st = CEP_INST_DONE;
      break;
    }
    t += a.dt;
    ++iout;
    if (!isfinite(y.V)) {
      st = CEP_INST_NONFINITE;
      break;
    }
  }
  M::template store<G>(y, a.y, a.ld, i);
  if (bm_on) bm::hot_store(a.bv, i, hot);
  a.t[i] = t;
  a.iout[i] = iout;
  a.status[i] = st;
}

// Warp-specialised form of run_kernel for populations too small to fill the
// GPU one thread per cell: a block of 4 warps advances 32 cells, warp r
// evaluating role r of the model (the channel groups of model_ord.cuh) for
// all 32. Each step the roles' contributions go through double-buffered
// shared memory ([2][4 roles][8 fields][32 cells], lane-contiguous, no bank
// conflicts) behind one barrier; every warp then applies the forward-Euler
// update of V and the ions to its own copy of those FP64 states (identical
// inputs and operations, so the copies stay identical) and warp 0 runs the
// biomarker state machine. The trip count is the same for every lane;
// finished or invalid lanes are predicated off so the barrier stays uniform.
template <class M, class P, int R, int R2 = -1>
__device__ __forceinline__ void role_loop(const RunArgs &a, typename P::G (*part)[4][8][32], int lane) {
  using G = typename P::G;
  const int64_t i = (int64_t)blockIdx.x * 32 + lane;
  const bool valid = i < a.n;
  const int64_t il = valid ? i : (int64_t)a.n - 1;
  int st = a.status[il];
  bool alive = valid && st == CEP_INST_RUNNING;
  if (!__syncthreads_or(alive)) return;  // uniform: every warp sees the same 32 cells
  typename M::template Y<G> y;
  typename M::template Par<G> q;
  M::template load<G>(y, a.y, a.ld, il);
  M::template load_par<G>(q, a.par, a.ld, il);
  double t = a.t[il];
  int iout = a.iout[il];
  const bm::Sched sc{a.sched[il], a.sched[a.ld + il], a.sched[2 * a.ld + il], a.sched[3 * a.ld + il]};
  const bool bm_on = R == 0 && a.bm_on && sc.first_pace >= 0;
  int cnt_print = bm::countdown(iout, sc.print_freq);
  int cnt_bcl = bm::countdown(iout, sc.steps_per_bcl);
  const double bcl = a.par[M::p_bcl() * a.ld + il];
  const double stim_start = a.par[M::p_stim_start() * a.ld + il];
  typename M::template Cur<G> c;
  bm::Hot hot;
  if (bm_on) bm::hot_load(a.bv, il, hot);
  int buf = 0;
  for (int k = 0; k <= a.n_steps; ++k) {
    const bool can_update = iout < sc.imax;
    const bool active = alive && !(can_update && k == a.n_steps);
    const bool upd = active && can_update;
    const double V0 = y.V;
    const double cai0 = M::cai_of(y);
    const auto ctx = ord::context<P>(y, q, t, a.stim_mode);
    {
      ord::Part<G> p;
      ord::role<P, M::kCipa, R>(y, q, ctx, a.dt, upd, p);
#pragma unroll
      for (int f = 0; f < 8; ++f) {
        const int fld = ord::role_field<ord::kIK1InNa<P>>(R, f);
        if (fld >= 0) part[buf][R][f][lane] = p.f[fld];
      }
    }
    if constexpr (R2 >= 0) {  // a warp that carries two channel groups
      ord::Part<G> p;
      ord::role<P, M::kCipa, R2>(y, q, ctx, a.dt, upd, p);
#pragma unroll
      for (int f = 0; f < 8; ++f) {
        const int fld = ord::role_field<ord::kIK1InNa<P>>(R2, f);
        if (fld >= 0) part[buf][R2][f][lane] = p.f[fld];
      }
    }
    __syncthreads();
    ord::Part<G> s;
#pragma unroll
    for (int f = 0; f < ord::kNumSums; ++f) s.f[f] = (G)0;
#pragma unroll
    for (int r = 0; r < 4; ++r) {
#pragma unroll
      for (int f = 0; f < 8; ++f) {
        const int fld = ord::role_field<ord::kIK1InNa<P>>(r, f);
        if (fld >= 0) s.f[fld] += part[buf][r][f][lane];
      }
    }
    ord::combine<P>(y, q, s, a.dt, upd, c);
    if (bm_on && active && iout >= 1)
      bm::sample(a.bv, i, sc, iout, t, a.dt, bcl, stim_start, V0, cai0, (double)c.dVdt, (double)c.INaL,
                 (double)c.ICaL, (double)c.Ito, (double)c.IKr, (double)c.IKs, (double)c.IK1, a.qnet_thr,
                 cnt_print, cnt_bcl, hot);
    if (active) {
      if (!can_update) {
        st = CEP_INST_DONE;
        alive = false;
      } else {
        t += a.dt;
        ++iout;
        if (!isfinite(y.V)) {
          st = CEP_INST_NONFINITE;
          alive = false;
        }
      }
    }
    buf ^= 1;
  }
  if (valid) {
    if (bm_on) bm::hot_store(a.bv, i, hot);
    ord::store_role<M::kCipa, ord::kIK1InNa<P>>(R, y, a.y, a.ld, i);
    if constexpr (R2 >= 0) ord::store_role<M::kCipa, ord::kIK1InNa<P>>(R2, y, a.y, a.ld, i);
    if (R == 0) {
      a.t[i] = t;
      a.iout[i] = iout;
      a.status[i] = st;
    }
  }
}

template <class M, class P>
__global__ void __launch_bounds__(128) run_roles_kernel(RunArgs a) {
  using G = typename P::G;
  __shared__ G part[2][4][8][32];
  const int lane = threadIdx.x & 31;
  const int role = pick_role();
  switch (role) {
    case 0: role_loop<M, P, 0>(a, part, lane); break;
    case 1: role_loop<M, P, 1>(a, part, lane); break;
    case 2: role_loop<M, P, 2>(a, part, lane); break;
    default: role_loop<M, P, 3>(a, part, lane); break;
  }
}

// Two warps per 32 cells, each carrying two channel groups (Na + Ca, K + the
// rest): half the warps of run_roles_kernel, twice the code per warp. Of the
// three pairings this one balanced the two warps best on the CiPA
// population (4.79e9 vs 4.49e9 cell-steps/s for Na + K | Ca + rest).
template <class M, class P>
__global__ void __launch_bounds__(64) run_pairs_kernel(RunArgs a) {
  using G = typename P::G;
  __shared__ G part[2][4][8][32];
  const int lane = threadIdx.x & 31;
  if ((threadIdx.x >> 5) == 0)
    role_loop<M, P, 0, 2>(a, part, lane);
  else
    role_loop<M, P, 1, 3>(a, part, lane);
}

// One Godunov ionic step of a tissue: every node advances by dt from the
// tissue clock t with the stimulus flag of its S1 mask window; no biomarker
// bookkeeping, so only the state and the parameters cross HBM.
struct TissueArgs {
  double *y;
  const double *par;
  int64_t ld;
  int n;
  double t, dt;
  const unsigned char *mask;  // null: stim_on is the mode of every instance
  int stim_on;  // the window test, uniform over the tissue (or -1/0/1 without a mask)
  const CepProto *proto;       // S1-S2 / ectopic state on the device, or null
  const unsigned char *mask2;  // ectopic region (with proto)
};

template <class M, class P>
__global__ void __launch_bounds__(128) tissue_kernel(TissueArgs a) {
  using G = typename P::G;
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  typename M::template Y<G> y;
  typename M::template Par<G> q;
  M::template load<G>(y, a.y, a.ld, i);
  M::template load_par<G>(q, a.par, a.ld, i);
  typename M::template Cur<G> c;
  int mode = a.mask ? ((a.stim_on && a.mask[i]) ? 1 : 0) : a.stim_on;
  if (a.proto) {  // S1 stays off once the protocol fired; the ectopic region as S1 (isEctopic)
    if (a.proto->fired && a.mask) mode = 0;
    if (a.mask2 && a.proto->ecto_on && a.mask2[i]) mode = 1;
  }
  M::template step<P>(y, q, a.t, a.dt, mode, true, c);
  M::template store<G>(y, a.y, a.ld, i);
}

// Dynamic restitution (apdr_bench.cpp:103-232): one thread per instance, a
// launch advances up to n_steps steps of the current BCL segment with the
// per-pace APD90 tracker in registers. The tracker and the segment clock
// persist between launches in rf/ri; the pace's Vm samples go to trace
// ([S][ld], coalesced) for the recalibration search at a boundary whose
// windowed peak stayed below 10 mV. The products and sums the reference
// writes as one expression are rounded separately (__dmul_rn/__dadd_rn) so
// no FMA contraction changes them.
enum : int { RF_peak = 0, RF_valley, RF_repol, RF_tpeak, RF_tdepol, RF_trepol, RF_apd, RF_t, RF_tp0, kRF };
enum : int { RI_repl = 0, RI_pace, RI_all, RI_iout, RI_nrec, RI_recal, RI_status, kRI };

struct RestitArgs {
  double *y;
  const double *par;
  int64_t ld;
  int n;
  double dt, bcl;
  int S, imax, n_steps;
  double *rf;      // [kRF][ld]
  int *ri;         // [kRI][ld]
  double *trace;   // [S][ld]
  cep_apdr_record_t *rec;  // [n][max_rec]
  int max_rec;
};

__global__ void restit_init_kernel(RestitArgs a) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  const int64_t ld = a.ld;
  const double v0 = a.y[i];
  for (int k = 0; k < kRF; ++k) a.rf[k * ld + i] = 0.0;
  for (int k = 0; k < kRI; ++k) a.ri[k * ld + i] = 0;
  a.rf[RF_peak * ld + i] = v0;  // vm_valley = vm_peak = STATES[V] (:97)
  a.rf[RF_valley * ld + i] = v0;
}

// Segment start (:111-130): the clock restarts, the tracker carries over.
__global__ void restit_segment_kernel(RestitArgs a) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  const int64_t ld = a.ld;
  a.rf[RF_t * ld + i] = 0.0;
  a.rf[RF_tp0 * ld + i] = 0.0;
  a.rf[RF_tdepol * ld + i] = 0.0;
  a.rf[RF_trepol * ld + i] = 0.0;
  a.ri[RI_iout * ld + i] = 0;
  a.ri[RI_pace * ld + i] = 0;
}

template <class M, class P>
__global__ void __launch_bounds__(128) restit_kernel(RestitArgs a) {
  using G = typename P::G;
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  const int64_t ld = a.ld;
  int st = a.ri[RI_status * ld + i];
  int iout = a.ri[RI_iout * ld + i];
  if (st != 0 || iout > a.imax) return;
  typename M::template Y<G> y;
  typename M::template Par<G> q;
  M::template load<G>(y, a.y, ld, i);
  M::template load_par<G>(q, a.par, ld, i);
  double vm_peak = a.rf[RF_peak * ld + i], vm_valley = a.rf[RF_valley * ld + i];
  double vm_repol = a.rf[RF_repol * ld + i], t_peak = a.rf[RF_tpeak * ld + i];
  double t_depol = a.rf[RF_tdepol * ld + i], t_repol = a.rf[RF_trepol * ld + i];
  double apd90 = a.rf[RF_apd * ld + i], t = a.rf[RF_t * ld + i], tp0 = a.rf[RF_tp0 * ld + i];
  int repl = a.ri[RI_repl * ld + i], pace = a.ri[RI_pace * ld + i], all_pace = a.ri[RI_all * ld + i];
  int n_rec = a.ri[RI_nrec * ld + i], recal = a.ri[RI_recal * ld + i];
  const double stim_start = a.par[M::p_stim_start() * ld + i];
  const double bcl = a.bcl, dt = a.dt;
  const int S = a.S;
  typename M::template Cur<G> c;
  for (int k = 0; k < a.n_steps && iout <= a.imax; ++k) {
    M::template step<P>(y, q, t, dt, -1, true, c);
    ++iout;
    t += dt;
    const double V = y.V;
    if (!isfinite(V)) {
      st = CEP_INST_NONFINITE;
      break;
    }
    const int j = iout - 1 - S * pace;  // sample index within the pace, in [0, S)
    a.trace[(int64_t)j * ld + i] = V;
    const double lo = __dadd_rn(__dmul_rn(bcl, (double)pace), stim_start);
    if (lo + 4. < t && t < lo + 56.) {  // :149-157
      if (vm_peak < V) {
        vm_peak = V;
        t_peak = t;
      }
    } else if (t > lo + 56.) {
      vm_repol = __dsub_rn(vm_peak, __dmul_rn(0.9, __dsub_rn(vm_peak, vm_valley)));
    }
    if (t > lo + 56. && vm_repol >= V && V > vm_repol - 2) {  // :161-166
      t_depol = lo;
      t_repol = t;
      apd90 = t_repol - t_depol;
      repl = 1;
    }
    if (iout % S == 0) {  // pace boundary :169-213
      if (vm_peak < 0 || (vm_peak >= 0 && vm_peak < 10)) {
        repl = 0;
        recal = 1;
        double tt = tp0;
        for (int jj = 0; jj < S; ++jj) {
          tt += dt;
          const double v = a.trace[(int64_t)jj * ld + i];
          if (vm_peak < v) {
            vm_peak = v;
            vm_repol = __dsub_rn(vm_peak, __dmul_rn(0.9, __dsub_rn(vm_peak, vm_valley)));
            t_peak = tt;
          }
        }
        tt = tp0;
        for (int jj = 0; jj < S; ++jj) {
          tt += dt;
          const double v = a.trace[(int64_t)jj * ld + i];
          if (tt > t_peak && vm_repol >= v && v > vm_repol - 1) {
            t_depol = lo;
            t_repol = tt;
            apd90 = t_repol - t_depol;
            repl = 1;
          }
        }
      }
      if (!repl) {
        t_depol = lo;
        t_repol = t;
        apd90 = t_repol - t_depol;
      }
      vm_valley = V;
      vm_peak = -999;
      vm_repol = 0;
      ++pace;
      ++all_pace;
      repl = 0;
      if (pace > 2) {
        if (n_rec < a.max_rec) {
          cep_apdr_record_t r;
          r.pace = all_pace;
          r.recal = recal;
          r.bcl = bcl;
          r.apd90 = apd90;
          r.di = (t + stim_start) - t_repol;
          r.t = t;
          a.rec[i * a.max_rec + n_rec] = r;
        }
        ++n_rec;
      }
      recal = 0;
      tp0 = t;
    }
  }
  M::template store<G>(y, a.y, ld, i);
  a.rf[RF_peak * ld + i] = vm_peak; a.rf[RF_valley * ld + i] = vm_valley; a.rf[RF_repol * ld + i] = vm_repol;
  a.rf[RF_tpeak * ld + i] = t_peak; a.rf[RF_tdepol * ld + i] = t_depol; a.rf[RF_trepol * ld + i] = t_repol;
  a.rf[RF_apd * ld + i] = apd90; a.rf[RF_t * ld + i] = t; a.rf[RF_tp0 * ld + i] = tp0;
  a.ri[RI_repl * ld + i] = repl; a.ri[RI_pace * ld + i] = pace; a.ri[RI_all * ld + i] = all_pace;
  a.ri[RI_iout * ld + i] = iout; a.ri[RI_nrec * ld + i] = n_rec; a.ri[RI_recal * ld + i] = recal;
  a.ri[RI_status * ld + i] = st;
}

// Voltage-clamp replay (CEPPatch/benchpatch.cpp:83-100): V set to v[k]
// before step k, the selected channel current of the step to out[k][ld].
struct ClampArgs {
  double *y;
  const double *par;
  int64_t ld;
  int n;
  const double *v;  // [m] clamp potentials of this chunk
  int m, current;
  double t0, dt;
  double *out;      // [m][ld]
};

template <class M, class P>
__global__ void __launch_bounds__(128) clamp_kernel(ClampArgs a) {
  using G = typename P::G;
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  typename M::template Y<G> y;
  typename M::template Par<G> q;
  M::template load<G>(y, a.y, a.ld, i);
  M::template load_par<G>(q, a.par, a.ld, i);
  typename M::template Cur<G> c;
  double t = a.t0;
  for (int k = 0; k < a.m; ++k) {
    y.V = a.v[k];
    M::template step<P>(y, q, t, a.dt, -1, true, c);
    double x;
    switch (a.current) {
      case 0: x = (double)c.INa; break;
      case 1: x = (double)c.INaL; break;
      case 2: x = (double)c.Ito; break;
      case 3: x = (double)c.ICaL; break;
      case 4: x = (double)c.IKr; break;
      case 5: x = (double)c.IKs; break;
      default: x = (double)c.IK1; break;
    }
    a.out[(int64_t)k * a.ld + i] = x;
    t += a.dt;
  }
  M::template store<G>(y, a.y, a.ld, i);
}

// Rates at the current state (no update).
template <class M>
__global__ void rates_kernel(const double *s, const double *par, int64_t ld, int n, double t, int stim_mode,
                             double *dvdt, double *cur) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  typename M::template Y<double> y;
  typename M::template Par<double> q;
  M::template load<double>(y, s, ld, i);
  M::template load_par<double>(q, par, ld, i);
  typename M::template Cur<double> c;
  M::template step<F64>(y, q, t, 0.0, stim_mode, false, c);
  if (dvdt) dvdt[i] = c.dVdt;
  if (cur) {
    cur[0 * (int64_t)n + i] = c.INa; cur[1 * (int64_t)n + i] = c.INaL; cur[2 * (int64_t)n + i] = c.Ito;
    cur[3 * (int64_t)n + i] = c.ICaL; cur[4 * (int64_t)n + i] = c.IKr; cur[5 * (int64_t)n + i] = c.IKs;
    cur[6 * (int64_t)n + i] = c.IK1;
  }
}

// The full RATES vector at the current state: one step under F64Rates
// leaves every state's right-hand side in its place; out[i][ns] (AoS).
template <class M>
__global__ void rates_all_kernel(const double *s, const double *par, int64_t ld, int n, double t, double *out) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  typename M::template Y<double> y;
  typename M::template Par<double> q;
  M::template load<double>(y, s, ld, i);
  M::template load_par<double>(q, par, ld, i);
  typename M::template Cur<double> c;
  M::template step<F64Rates>(y, q, t, 0.0, -1, true, c);
  double tmp[64];
  M::template store<double>(y, tmp, 1, 0);  // state order, stride 1
  for (int k = 0; k < M::kStates; ++k) out[i * M::kStates + k] = tmp[k];
}

__global__ void collect_bm_kernel(bm::View v, const int *status, int64_t first, int count, cep_biomarkers_t *out) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= count) return;
  const int64_t i = first + k;
  cep_biomarkers_t r;
  const int S = bm::F_S0;
  r.qnet = v.F(S + bm::B_qnet, i) / 1000.0;
  r.inal_auc = v.F(S + bm::B_inal, i);
  r.ical_auc = v.F(S + bm::B_ical, i);
  r.dvmdt_repol = v.F(S + bm::B_dvmdt_repol, i);
  r.dvmdt_max = v.F(S + bm::B_dvmdt_max, i);
  r.vm_peak = v.F(S + bm::B_vm_peak, i);
  r.vm_valley = v.F(S + bm::B_vm_valley, i);
  r.vm_dia = v.F(S + bm::B_vm_dia, i);
  r.apd90 = v.F(S + bm::B_apd90, i);
  r.apd50 = v.F(S + bm::B_apd50, i);
  r.apd_tri = r.apd90 - r.apd50;
  r.ca_peak = v.F(S + bm::B_ca_peak, i);
  r.ca_valley = v.F(S + bm::B_ca_valley, i);
  r.ca_dia = v.F(S + bm::B_ca_dia, i);
  r.cad90 = v.F(S + bm::B_cad90, i);
  r.cad50 = v.F(S + bm::B_cad50, i);
  r.cad_tri = r.cad90 - r.cad50;
  r.steepest_pace = v.I(bm::I_steepest, i);
  r.n_eligible = v.I(bm::I_n_elig, i);
  r.status = status[i];
  r.reserved = 0;
  out[k] = r;
}

// ------------------------------------------------------------- dispatch
template <class M>
struct Ops {
  static int launch_init(cep_batch *b, int64_t first, int count, const double *ct, const double *conc,
                         const double *hill, int hs, unsigned flags) {
    const int grid = (count + kBlock - 1) / kBlock;
    init_kernel<M><<<grid, kBlock, 0, b->stream>>>(b->params, b->states, b->ld, first, count, ct, conc, hill, hs,
                                                   flags);
    return cudaGetLastError() == cudaSuccess ? CEP_OK : fail(CEP_ERR_CUDA, "init launch failed");
  }
  static int launch_pacing(cep_batch *b, int64_t first, int count, double bcl, double start, double dur,
                           double amp) {
    const int grid = (count + kBlock - 1) / kBlock;
    pacing_kernel<<<grid, kBlock, 0, b->stream>>>(b->params, b->ld, first, count, M::p_bcl(), M::p_stim_start(),
                                                  M::p_duration(), M::p_amp(), bcl, start, dur, amp);
    return cudaGetLastError() == cudaSuccess ? CEP_OK : fail(CEP_ERR_CUDA, "pacing launch failed");
  }
  static int launch_reset(cep_batch *b, const RunArgs &a, int64_t first, int count) {
    const int grid = (count + kBlock - 1) / kBlock;
    reset_kernel<<<grid, kBlock, 0, b->stream>>>(a, first, count, M::p_bcl(), M::p_stim_start(), M::kCai);
    return cudaGetLastError() == cudaSuccess ? CEP_OK : fail(CEP_ERR_CUDA, "reset launch failed");
  }
  static int launch_run(cep_batch *b, const RunArgs &a) {
    if constexpr (std::is_same<M, Tt06Model>::value || std::is_same<M, Tt04Model>::value ||
                  std::is_same<M, TomekModel>::value) {
      const int block = b->block;
      const int grid = (b->n + block - 1) / block;
      if (b->precision == CEP_PREC_MIXED)
        run_kernel<M, Mixed><<<grid, block, 0, b->stream>>>(a);
      else
        run_kernel<M, F64><<<grid, block, 0, b->stream>>>(a);
    } else if (b->variant == CEP_KERNEL_ROLES) {
      const int grid = (b->n + 31) / 32;
      if (b->precision == CEP_PREC_MIXED)
        run_roles_kernel<M, Mixed><<<grid, 128, 0, b->stream>>>(a);
      else
        run_roles_kernel<M, F64><<<grid, 128, 0, b->stream>>>(a);
    } else if (b->variant == CEP_KERNEL_PAIRS) {
      const int grid = (b->n + 31) / 32;
      if (b->precision == CEP_PREC_MIXED)
        run_pairs_kernel<M, Mixed><<<grid, 64, 0, b->stream>>>(a);
      else
        run_pairs_kernel<M, F64><<<grid, 64, 0, b->stream>>>(a);
    } else {
      const int block = b->block;
      const int grid = (b->n + block - 1) / block;
      if (b->precision == CEP_PREC_MIXED)
        run_kernel<M, Mixed><<<grid, block, 0, b->stream>>>(a);
      else
        run_kernel<M, F64><<<grid, block, 0, b->stream>>>(a);
    }
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? CEP_OK : fail(CEP_ERR_CUDA, "run launch failed: %s", cudaGetErrorString(e));
  }
  static int launch_tissue(cep_batch *b, const TissueArgs &a) {
    const int grid = (b->n + 127) / 128;
    if (b->precision == CEP_PREC_MIXED)
      tissue_kernel<M, Mixed><<<grid, 128, 0, b->stream>>>(a);
    else
      tissue_kernel<M, F64><<<grid, 128, 0, b->stream>>>(a);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? CEP_OK : fail(CEP_ERR_CUDA, "tissue launch failed: %s", cudaGetErrorString(e));
  }
  static int launch_restit(cep_batch *b, const RestitArgs &a) {
    const int grid = (b->n + 127) / 128;
    if (b->precision == CEP_PREC_MIXED)
      restit_kernel<M, Mixed><<<grid, 128, 0, b->stream>>>(a);
    else
      restit_kernel<M, F64><<<grid, 128, 0, b->stream>>>(a);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? CEP_OK : fail(CEP_ERR_CUDA, "restitution launch failed: %s", cudaGetErrorString(e));
  }
  static int launch_clamp(cep_batch *b, const ClampArgs &a) {
    const int grid = (b->n + 127) / 128;
    if (b->precision == CEP_PREC_MIXED)
      clamp_kernel<M, Mixed><<<grid, 128, 0, b->stream>>>(a);
    else
      clamp_kernel<M, F64><<<grid, 128, 0, b->stream>>>(a);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? CEP_OK : fail(CEP_ERR_CUDA, "clamp launch failed: %s", cudaGetErrorString(e));
  }
  static int launch_rates_all(cep_batch *b, double t, double *out) {
    if constexpr (M::kHasRates) {
      const int grid = (b->n + kBlock - 1) / kBlock;
      rates_all_kernel<M><<<grid, kBlock, 0, b->stream>>>(b->states, b->params, b->ld, b->n, t, out);
      return cudaGetLastError() == cudaSuccess ? CEP_OK : fail(CEP_ERR_CUDA, "rates launch failed");
    } else {
      (void)t; (void)out;
      return fail(CEP_ERR_UNSUPPORTED, "model %d integrates with its own fixed-step scheme only (no RATES vector)",
                  b->model);
    }
  }
  static int launch_rates(cep_batch *b, double t, double *dvdt, double *cur) {
    const int grid = (b->n + kBlock - 1) / kBlock;
    rates_kernel<M><<<grid, kBlock, 0, b->stream>>>(b->states, b->params, b->ld, b->n, t, -1, dvdt, cur);
    return cudaGetLastError() == cudaSuccess ? CEP_OK : fail(CEP_ERR_CUDA, "rates launch failed");
  }
};

struct ModelInfo {
  int ns, np, cai;
  int (*init)(cep_batch *, int64_t, int, const double *, const double *, const double *, int, unsigned);
  int (*pacing)(cep_batch *, int64_t, int, double, double, double, double);
  int (*reset)(cep_batch *, const RunArgs &, int64_t, int);
  int (*run)(cep_batch *, const RunArgs &);
  int (*rates)(cep_batch *, double, double *, double *);
  int p_bcl;
  int (*tissue)(cep_batch *, const TissueArgs &);
  int (*restit)(cep_batch *, const RestitArgs &);
  int (*clamp)(cep_batch *, const ClampArgs &);
  int (*rates_all)(cep_batch *, double, double *);
};

const ModelInfo *model_info(int model) {
  static const ModelInfo ord_info{OrdModel::kStates, OrdModel::kParams, OrdModel::kCai,
                                  &Ops<OrdModel>::launch_init, &Ops<OrdModel>::launch_pacing,
                                  &Ops<OrdModel>::launch_reset, &Ops<OrdModel>::launch_run,
                                  &Ops<OrdModel>::launch_rates, OrdModel::p_bcl(), &Ops<OrdModel>::launch_tissue,
                                  &Ops<OrdModel>::launch_restit, &Ops<OrdModel>::launch_clamp,
                                  &Ops<OrdModel>::launch_rates_all};
  static const ModelInfo cipa_info{CipaModel::kStates, CipaModel::kParams, CipaModel::kCai,
                                   &Ops<CipaModel>::launch_init, &Ops<CipaModel>::launch_pacing,
                                   &Ops<CipaModel>::launch_reset, &Ops<CipaModel>::launch_run,
                                   &Ops<CipaModel>::launch_rates, CipaModel::p_bcl(), &Ops<CipaModel>::launch_tissue,
                                  &Ops<CipaModel>::launch_restit, &Ops<CipaModel>::launch_clamp,
                                  &Ops<CipaModel>::launch_rates_all};
  static const ModelInfo tt06_info{Tt06Model::kStates, Tt06Model::kParams, Tt06Model::kCai,
                                   &Ops<Tt06Model>::launch_init, &Ops<Tt06Model>::launch_pacing,
                                   &Ops<Tt06Model>::launch_reset, &Ops<Tt06Model>::launch_run,
                                   &Ops<Tt06Model>::launch_rates, Tt06Model::p_bcl(), &Ops<Tt06Model>::launch_tissue,
                                  &Ops<Tt06Model>::launch_restit, &Ops<Tt06Model>::launch_clamp,
                                  &Ops<Tt06Model>::launch_rates_all};
  static const ModelInfo tomek_info{TomekModel::kStates, TomekModel::kParams, TomekModel::kCai,
                                   &Ops<TomekModel>::launch_init, &Ops<TomekModel>::launch_pacing,
                                   &Ops<TomekModel>::launch_reset, &Ops<TomekModel>::launch_run,
                                   &Ops<TomekModel>::launch_rates, TomekModel::p_bcl(), &Ops<TomekModel>::launch_tissue,
                                  &Ops<TomekModel>::launch_restit, &Ops<TomekModel>::launch_clamp,
                                  &Ops<TomekModel>::launch_rates_all};
  static const ModelInfo tt04_info{Tt04Model::kStates, Tt04Model::kParams, Tt04Model::kCai,
                                   &Ops<Tt04Model>::launch_init, &Ops<Tt04Model>::launch_pacing,
                                   &Ops<Tt04Model>::launch_reset, &Ops<Tt04Model>::launch_run,
                                   &Ops<Tt04Model>::launch_rates, Tt04Model::p_bcl(), &Ops<Tt04Model>::launch_tissue,
                                  &Ops<Tt04Model>::launch_restit, &Ops<Tt04Model>::launch_clamp,
                                  &Ops<Tt04Model>::launch_rates_all};
  switch (model) {
    case CEP_MODEL_TT2006: return &tt06_info;
    case CEP_MODEL_TT2004: return &tt04_info;
    case CEP_MODEL_TOMEK2019: return &tomek_info;
    case CEP_MODEL_ORD2011: return &ord_info;
    case CEP_MODEL_CIPA2017: return &cipa_info;
    default: return nullptr;
  }
}

}  // namespace cep

using namespace cep;

namespace {

template <class T>
int dev_alloc(cep_batch *b, T **p, size_t count) {
  void *q = nullptr;
  const cudaError_t e = cudaMalloc(&q, count * sizeof(T) + 256);
  if (e != cudaSuccess) return fail(CEP_ERR_OOM, "cudaMalloc(%zu bytes): %s", count * sizeof(T), cudaGetErrorString(e));
  b->allocs.push_back(q);
  *p = static_cast<T *>(q);
  return CEP_OK;
}

RunArgs make_args(cep_batch *b, long n_steps) {
  RunArgs a;
  a.y = b->states; a.par = b->params; a.ld = b->ld; a.n = b->n; a.t = b->t; a.iout = b->iout;
  a.status = b->status; a.sched = b->sched; a.dt = b->dt; a.n_steps = (int)n_steps;
  a.bm_on = (b->bmf != nullptr && b->first_pace >= 0) ? 1 : 0;
  a.bv.f = b->bmf; a.bv.fi = b->bmi; a.bv.ca_t = b->ca_t; a.bv.ca_v = b->ca_v; a.bv.ca_cap = b->ca_cap;
  a.bv.ld = b->ld;
  a.qnet_thr = b->qnet_thr;
  a.stim_mode = -1;
  return a;
}

}  // namespace

extern "C" {

const char *cep_version(void) { return "cep_b200 0.1 (sm_100a)"; }
const char *cep_last_error(void) { return g_last_error.c_str(); }

int cep_device_count(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

int cep_batch_create(int model, int n, int precision, void *stream, cep_batch_t *out) {
  if (!out) return fail(CEP_ERR_ARG, "out is NULL");
  *out = nullptr;
  if (n <= 0) return fail(CEP_ERR_ARG, "n must be positive (got %d)", n);
  if (precision != CEP_PREC_FP64 && precision != CEP_PREC_MIXED) return fail(CEP_ERR_ARG, "bad precision %d", precision);
  const ModelInfo *mi = model_info(model);
  if (!mi) return fail(CEP_ERR_UNSUPPORTED, "model %d not built", model);
  if (cep_device_count() == 0) return fail(CEP_ERR_NO_DEVICE, "no CUDA device visible");
  cep_batch *b = new cep_batch();
  b->model = model; b->n = n; b->ns = mi->ns; b->np = mi->np; b->precision = precision;
  b->ld = ((int64_t)n + 31) / 32 * 32;
  b->stream = static_cast<cudaStream_t>(stream);
  // Launch shape: the run kernels hold ~250 registers per thread, so an SM
  // keeps at most 8 warps. A population smaller than the GPU's resident
  // capacity is spread as 1-warp blocks so that every SM gets work.
  {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    b->block = (n <= sms * 8 * 32) ? 32 : 128;
    // Below ~1.5 waves of one-thread-per-cell occupancy the warp-specialised
    // kernels keep more warps in flight. Measured on the CiPA population
    // (us per step; cell / 4 roles / 2 pairs): mixed, 10,000 instances
    // 2.90 / 2.47 / 2.16, 320 instances 2.69 / 1.38 / 1.71; FP64 (exp and
    // log out of line), 10,000 instances 22.2 / 9.5 / 11.7, 320 instances
    // 21.5 / 7.2 / 11.1. So FP64 takes the four roles, mixed the four roles
    // up to one 32-cell group per SM and the pairs above.
    const bool ord_family = model == CEP_MODEL_ORD2011 || model == CEP_MODEL_CIPA2017;
    if (!ord_family || n > sms * 12 * 32)
      b->variant = CEP_KERNEL_CELL;
    else if (precision == CEP_PREC_FP64 || n <= sms * 32)
      b->variant = CEP_KERNEL_ROLES;
    else
      b->variant = CEP_KERNEL_PAIRS;
  }
  int rc = CEP_OK;
  if ((rc = dev_alloc(b, &b->states, (size_t)b->ns * b->ld)) || (rc = dev_alloc(b, &b->params, (size_t)b->np * b->ld)) ||
      (rc = dev_alloc(b, &b->t, (size_t)b->ld)) || (rc = dev_alloc(b, &b->iout, (size_t)b->ld)) ||
      (rc = dev_alloc(b, &b->status, (size_t)b->ld)) || (rc = dev_alloc(b, &b->sched, (size_t)4 * b->ld))) {
    cep_batch_destroy(b);
    return rc;
  }
  cudaMemsetAsync(b->t, 0, sizeof(double) * b->ld, b->stream);
  cudaMemsetAsync(b->iout, 0, sizeof(int) * b->ld, b->stream);
  cudaMemsetAsync(b->status, 0, sizeof(int) * b->ld, b->stream);
  // default schedule: unbounded run, biomarkers off
  std::vector<int> sc((size_t)4 * b->ld, 0);
  for (int64_t i = 0; i < b->ld; ++i) { sc[i] = 0x7fffffff; sc[3 * b->ld + i] = -1; }
  if (copy_sync(b->sched, sc.data(), sc.size() * sizeof(int), cudaMemcpyHostToDevice, b->stream) != CEP_OK) {
    cep_batch_destroy(b);
    return fail(CEP_ERR_CUDA, "schedule upload failed");
  }
  *out = b;
  return CEP_OK;
}

int cep_batch_destroy(cep_batch_t b) {
  if (!b) return CEP_OK;
  if (b->stream) cudaStreamSynchronize(b->stream); else cudaDeviceSynchronize();
  for (void *p : b->allocs) cudaFree(p);
  delete b;
  return CEP_OK;
}

int cep_batch_set_block(cep_batch_t b, int threads_per_block) {
  if (!b) return fail(CEP_ERR_ARG, "null batch");
  if (threads_per_block != 32 && threads_per_block != 64 && threads_per_block != 96 && threads_per_block != 128)
    return fail(CEP_ERR_ARG, "threads_per_block must be 32, 64, 96 or 128");
  b->block = threads_per_block;
  return CEP_OK;
}

int cep_batch_set_kernel(cep_batch_t b, int variant) {
  if (!b) return fail(CEP_ERR_ARG, "null batch");
  if (variant != CEP_KERNEL_CELL && variant != CEP_KERNEL_ROLES && variant != CEP_KERNEL_PAIRS)
    return fail(CEP_ERR_ARG, "bad kernel variant %d", variant);
  if (variant != CEP_KERNEL_CELL && b->model != CEP_MODEL_ORD2011 && b->model != CEP_MODEL_CIPA2017)
    return fail(CEP_ERR_UNSUPPORTED, "warp-specialised kernel exists for the ORd family only");
  b->variant = variant;
  return CEP_OK;
}

int cep_batch_autotune(cep_batch_t b, long n_steps, int *variant_out, int *block_out) {
  if (!b) return fail(CEP_ERR_ARG, "null batch");
  if (!b->initialized) return fail(CEP_ERR_STATE, "cep_batch_init must come first");
  if (n_steps <= 0) n_steps = 400;
  if (n_steps > 100000) return fail(CEP_ERR_ARG, "n_steps out of range (1..100000)");
  // everything a run launch writes, saved once and put back before each
  // trial and at the end
  struct Region {
    void *p;
    size_t bytes;
    void *save;
  };
  std::vector<Region> regions = {{b->states, sizeof(double) * (size_t)b->ns * b->ld, nullptr},
                                 {b->t, sizeof(double) * (size_t)b->ld, nullptr},
                                 {b->iout, sizeof(int) * (size_t)b->ld, nullptr},
                                 {b->status, sizeof(int) * (size_t)b->ld, nullptr}};
  if (b->bmf) {
    regions.push_back({b->bmf, sizeof(double) * (size_t)bm::kNumF * b->ld, nullptr});
    regions.push_back({b->bmi, sizeof(int) * (size_t)bm::kNumI * b->ld, nullptr});
  }
  if (b->ca_t) {
    regions.push_back({b->ca_t, sizeof(double) * (size_t)b->ca_cap * b->ld, nullptr});
    regions.push_back({b->ca_v, sizeof(double) * (size_t)b->ca_cap * b->ld, nullptr});
  }
  struct Saved {
    std::vector<Region> *r;
    ~Saved() {
      for (Region &g : *r)
        if (g.save) cudaFree(g.save);
    }
  } saved{&regions};
  for (Region &g : regions) {
    if (cudaMalloc(&g.save, g.bytes) != cudaSuccess) {
      cudaGetLastError();
      g.save = nullptr;
      return fail(CEP_ERR_OOM, "autotune: no room to save %zu bytes of batch state", g.bytes);
    }
    CEP_CUDA(cudaMemcpyAsync(g.save, g.p, g.bytes, cudaMemcpyDeviceToDevice, b->stream));
  }
  auto restore = [&]() -> int {
    for (Region &g : regions) CEP_CUDA(cudaMemcpyAsync(g.p, g.save, g.bytes, cudaMemcpyDeviceToDevice, b->stream));
    return CEP_OK;
  };
  struct Cand {
    int variant, block;
  };
  std::vector<Cand> cands = {{CEP_KERNEL_CELL, 32}, {CEP_KERNEL_CELL, 64}, {CEP_KERNEL_CELL, 128}};
  if (b->model == CEP_MODEL_ORD2011 || b->model == CEP_MODEL_CIPA2017) {
    cands.push_back({CEP_KERNEL_PAIRS, b->block});
    cands.push_back({CEP_KERNEL_ROLES, b->block});
  }
  const int keep_variant = b->variant, keep_block = b->block;
  cudaEvent_t e0, e1;
  CEP_CUDA(cudaEventCreate(&e0));
  CEP_CUDA(cudaEventCreate(&e1));
  float best_ms = 1e30f;
  Cand best{keep_variant, keep_block};
  int rc = CEP_OK;
  const ModelInfo *mi = model_info(b->model);
  for (const Cand &c : cands) {
    b->variant = c.variant;
    b->block = c.block;
    RunArgs a = make_args(b, n_steps);
    if (!b->has_protocol) a.bm_on = 0;
    // one untimed launch (code and caches warm), then the timed one, both
    // from the saved state
    if ((rc = restore()) || (rc = mi->run(b, a)) || (rc = restore())) break;
    if (cudaEventRecord(e0, b->stream) != cudaSuccess || (rc = mi->run(b, a)) ||
        cudaEventRecord(e1, b->stream) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess) {
      if (!rc) rc = fail(CEP_ERR_CUDA, "autotune trial failed");
      break;
    }
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (ms < best_ms) {
      best_ms = ms;
      best = c;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  const int rc2 = restore();
  const cudaError_t e = cudaStreamSynchronize(b->stream);
  if (rc || rc2 || e != cudaSuccess) {
    b->variant = keep_variant;
    b->block = keep_block;
    return rc ? rc : rc2 ? rc2 : fail(CEP_ERR_CUDA, "autotune: %s", cudaGetErrorString(e));
  }
  b->variant = best.variant;
  b->block = best.block;
  if (variant_out) *variant_out = best.variant;
  if (block_out) *block_out = best.block;
  return CEP_OK;
}

// ------------------------------------------------------------ checkpoint
// Blob layout: CkptHeader, then each device array in the order of
// ckpt_regions(), each the full [rows][ld] block.
namespace {
struct CkptHeader {
  char magic[8];  // "CEPBATC1"
  int32_t model, n, ns, np, precision, ca_cap, n_pace, first_pace, variant, block;
  int32_t initialized, has_protocol, has_bm, reserved;
  int64_t ld;
  double dt, dt_write, qnet_thr;
};
struct CkptRegion {
  void *p;
  size_t bytes;
};
std::vector<CkptRegion> ckpt_regions(const cep_batch *b, bool has_bm, int ca_cap) {
  std::vector<CkptRegion> r = {{b->states, sizeof(double) * (size_t)b->ns * b->ld},
                               {b->params, sizeof(double) * (size_t)b->np * b->ld},
                               {b->t, sizeof(double) * (size_t)b->ld},
                               {b->iout, sizeof(int) * (size_t)b->ld},
                               {b->status, sizeof(int) * (size_t)b->ld},
                               {b->sched, sizeof(int) * (size_t)4 * b->ld}};
  if (has_bm) {
    r.push_back({b->bmf, sizeof(double) * (size_t)bm::kNumF * b->ld});
    r.push_back({b->bmi, sizeof(int) * (size_t)bm::kNumI * b->ld});
  }
  if (ca_cap > 0) {
    r.push_back({b->ca_t, sizeof(double) * (size_t)ca_cap * b->ld});
    r.push_back({b->ca_v, sizeof(double) * (size_t)ca_cap * b->ld});
  }
  return r;
}
}  // namespace

int cep_batch_checkpoint_size(cep_batch_t b, size_t *bytes) {
  if (!b || !bytes) return fail(CEP_ERR_ARG, "null argument");
  size_t total = sizeof(CkptHeader);
  for (const CkptRegion &g : ckpt_regions(b, b->bmf != nullptr, b->ca_t ? b->ca_cap : 0)) total += g.bytes;
  *bytes = total;
  return CEP_OK;
}

int cep_batch_checkpoint(cep_batch_t b, void *buf, size_t bytes) {
  if (!b || !buf) return fail(CEP_ERR_ARG, "null argument");
  size_t need = 0;
  int rc = cep_batch_checkpoint_size(b, &need);
  if (rc) return rc;
  if (bytes < need) return fail(CEP_ERR_ARG, "checkpoint buffer has %zu bytes, needs %zu", bytes, need);
  CkptHeader h;
  std::memset(&h, 0, sizeof(h));
  std::memcpy(h.magic, "CEPBATC1", 8);
  h.model = b->model; h.n = b->n; h.ns = b->ns; h.np = b->np; h.precision = b->precision;
  h.ca_cap = b->ca_t ? b->ca_cap : 0; h.n_pace = b->n_pace; h.first_pace = b->first_pace;
  h.variant = b->variant; h.block = b->block; h.initialized = b->initialized; h.has_protocol = b->has_protocol;
  h.has_bm = b->bmf != nullptr; h.ld = b->ld; h.dt = b->dt; h.dt_write = b->dt_write; h.qnet_thr = b->qnet_thr;
  char *out = static_cast<char *>(buf);
  std::memcpy(out, &h, sizeof(h));
  size_t off = sizeof(h);
  for (const CkptRegion &g : ckpt_regions(b, h.has_bm, h.ca_cap)) {
    CEP_CUDA(cudaMemcpyAsync(out + off, g.p, g.bytes, cudaMemcpyDeviceToHost, b->stream));
    off += g.bytes;
  }
  CEP_CUDA(cudaStreamSynchronize(b->stream));
  return CEP_OK;
}

int cep_batch_restore(cep_batch_t b, const void *buf, size_t bytes) {
  if (!b || !buf) return fail(CEP_ERR_ARG, "null argument");
  if (bytes < sizeof(CkptHeader)) return fail(CEP_ERR_ARG, "checkpoint too short");
  CkptHeader h;
  std::memcpy(&h, buf, sizeof(h));
  if (std::memcmp(h.magic, "CEPBATC1", 8) != 0) return fail(CEP_ERR_ARG, "not a batch checkpoint");
  if (h.model != b->model || h.n != b->n || h.precision != b->precision || h.ld != b->ld || h.ns != b->ns ||
      h.np != b->np)
    return fail(CEP_ERR_ARG, "checkpoint of model %d, %d instances, precision %d does not fit this batch", h.model,
                h.n, h.precision);
  if (h.ca_cap < 0 || h.ca_cap > (1 << 24)) return fail(CEP_ERR_ARG, "corrupt checkpoint header");
  {  // the blob must hold every region its header announces before anything of the batch changes
    const size_t ld = (size_t)b->ld;
    size_t need = sizeof(CkptHeader) + ld * (sizeof(double) * ((size_t)b->ns + b->np + 1) + sizeof(int) * 6);
    if (h.has_bm) need += ld * (sizeof(double) * bm::kNumF + sizeof(int) * bm::kNumI);
    need += ld * sizeof(double) * 2 * (size_t)h.ca_cap;
    if (bytes < need) return fail(CEP_ERR_ARG, "checkpoint has %zu bytes, needs %zu", bytes, need);
  }
  int rc;
  if (h.has_bm && !b->bmf &&
      ((rc = dev_alloc(b, &b->bmf, (size_t)bm::kNumF * b->ld)) || (rc = dev_alloc(b, &b->bmi, (size_t)bm::kNumI * b->ld))))
    return rc;
  if (h.ca_cap > 0 && (!b->ca_t || b->ca_cap != h.ca_cap)) {
    if ((rc = dev_alloc(b, &b->ca_t, (size_t)h.ca_cap * b->ld)) || (rc = dev_alloc(b, &b->ca_v, (size_t)h.ca_cap * b->ld)))
      return rc;
  }
  b->ca_cap = h.ca_cap > 0 ? h.ca_cap : b->ca_cap;
  size_t need = sizeof(CkptHeader);
  const std::vector<CkptRegion> regs = ckpt_regions(b, h.has_bm, h.ca_cap);
  for (const CkptRegion &g : regs) need += g.bytes;
  if (bytes < need) return fail(CEP_ERR_ARG, "checkpoint has %zu bytes, needs %zu", bytes, need);
  const char *in = static_cast<const char *>(buf);
  size_t off = sizeof(CkptHeader);
  for (const CkptRegion &g : regs) {
    CEP_CUDA(cudaMemcpyAsync(g.p, in + off, g.bytes, cudaMemcpyHostToDevice, b->stream));
    off += g.bytes;
  }
  CEP_CUDA(cudaStreamSynchronize(b->stream));
  b->n_pace = h.n_pace; b->first_pace = h.first_pace; b->variant = h.variant; b->block = h.block;
  b->initialized = h.initialized != 0; b->has_protocol = h.has_protocol != 0;
  b->dt = h.dt; b->dt_write = h.dt_write; b->qnet_thr = h.qnet_thr;
  return CEP_OK;
}

int cep_batch_size(cep_batch_t b, int *n, int *n_states) {
  if (!b) return fail(CEP_ERR_ARG, "null batch");
  if (n) *n = b->n;
  if (n_states) *n_states = b->ns;
  return CEP_OK;
}

int cep_batch_init(cep_batch_t b, const double *celltype, const double *conc, const double *hill, int hill_stride,
                   unsigned flags) {
  if (!b) return fail(CEP_ERR_ARG, "null batch");
  if (hill && hill_stride < 14) return fail(CEP_ERR_ARG, "hill_stride must be >= 14 (got %d)", hill_stride);
  if ((flags & CEP_FLAG_NEO_ORD) && b->model != CEP_MODEL_ORD2011)
    return fail(CEP_ERR_UNSUPPORTED, "CEP_FLAG_NEO_ORD selects a build of ORd 2011 only");
  if ((flags & CEP_FLAG_NEO_ORD) && (flags & CEP_FLAG_QUIRKS))
    return fail(CEP_ERR_ARG, "CEP_FLAG_NEO_ORD and CEP_FLAG_QUIRKS name two different builds");
  const ModelInfo *mi = model_info(b->model);
  const int n = b->n;
  // validate the drug inputs on the host: NaN/negative IC50 rows are rejected
  if (conc)
    for (int i = 0; i < n; ++i)
      if (!(conc[i] >= 0.0) || !std::isfinite(conc[i])) return fail(CEP_ERR_ARG, "conc[%d] = %g is not a finite non-negative value", i, conc[i]);
  if (hill)
    for (int i = 0; i < n; ++i)
      for (int k = 0; k < hill_stride; ++k)
        if (!std::isfinite(hill[(size_t)i * hill_stride + k]) || hill[(size_t)i * hill_stride + k] < 0.0)
          if (k < 14) return fail(CEP_ERR_ARG, "hill[%d][%d] = %g is not a finite non-negative value", i, k, hill[(size_t)i * hill_stride + k]);
  double *d_ct = nullptr, *d_conc = nullptr, *d_hill = nullptr;
  const size_t bytes_h = hill ? (size_t)n * hill_stride * sizeof(double) : 0;
  CEP_CUDA(cudaMallocAsync((void **)&d_ct, sizeof(double) * n * 2 + bytes_h + 64, b->stream));
  d_conc = d_ct + n;
  d_hill = hill ? d_conc + n : nullptr;
  std::vector<double> zeros;
  if (!celltype || !conc) zeros.assign(n, 0.0);
  CEP_CUDA(cudaMemcpyAsync(d_ct, celltype ? celltype : zeros.data(), sizeof(double) * n, cudaMemcpyHostToDevice, b->stream));
  CEP_CUDA(cudaMemcpyAsync(d_conc, conc ? conc : zeros.data(), sizeof(double) * n, cudaMemcpyHostToDevice, b->stream));
  if (hill) CEP_CUDA(cudaMemcpyAsync(d_hill, hill, bytes_h, cudaMemcpyHostToDevice, b->stream));
  int rc = mi->init(b, 0, b->n, d_ct, d_conc, d_hill, hill_stride, flags);
  CEP_CUDA(cudaFreeAsync(d_ct, b->stream));
  CEP_CUDA(cudaStreamSynchronize(b->stream));
  if (rc) return rc;
  b->initialized = true;
  return CEP_OK;
}

int cep_batch_set_pacing(cep_batch_t b, double bcl, double stim_start, double stim_dur, double amp_scale) {
  if (!b) return fail(CEP_ERR_ARG, "null batch");
  if (!b->initialized) return fail(CEP_ERR_STATE, "cep_batch_init must come first");
  if (!(bcl > 0) || !std::isfinite(bcl)) return fail(CEP_ERR_ARG, "bcl must be positive");
  return model_info(b->model)->pacing(b, 0, b->n, bcl, stim_start, stim_dur, amp_scale);
}

// Parameter row of a scalable conductance for a model, or -1.
static int scale_param_index(int model, int g) {
  using namespace cep;
  switch (model) {
    case CEP_MODEL_ORD2011:
    case CEP_MODEL_CIPA2017:
      switch (g) {
        case CEP_SCALE_GNA: return ord::P_GNa; case CEP_SCALE_GNAL: return ord::P_GNaL;
        case CEP_SCALE_GTO: return ord::P_Gto; case CEP_SCALE_GCAL: return ord::P_PCa;
        case CEP_SCALE_GKR: return ord::P_GKr; case CEP_SCALE_GKS: return ord::P_GKs;
        case CEP_SCALE_GK1: return ord::P_GK1; case CEP_SCALE_GKB: return ord::P_GKb;
        case CEP_SCALE_GNCX: return ord::P_Gncx; case CEP_SCALE_PNAK: return ord::P_Pnak;
        default: return -1;
      }
    case CEP_MODEL_TOMEK2019:
      switch (g) {
        case CEP_SCALE_GNA: return tomek::P_GNa; case CEP_SCALE_GNAL: return tomek::P_GNaL;
        case CEP_SCALE_GTO: return tomek::P_Gto; case CEP_SCALE_GCAL: return tomek::P_PCa;
        case CEP_SCALE_GKR: return tomek::P_GKr; case CEP_SCALE_GKS: return tomek::P_GKs;
        case CEP_SCALE_GK1: return tomek::P_GK1; case CEP_SCALE_GKB: return tomek::P_GKb;
        case CEP_SCALE_GNCX: return tomek::P_Gncx; case CEP_SCALE_PNAK: return tomek::P_Pnak;
        default: return -1;
      }
    case CEP_MODEL_TT2006:
      switch (g) {
        case CEP_SCALE_GNA: return tt06::P_gNa; case CEP_SCALE_GTO: return tt06::P_gto;
        case CEP_SCALE_GCAL: return tt06::P_gCaL; case CEP_SCALE_GKR: return tt06::P_gKr;
        case CEP_SCALE_GKS: return tt06::P_gKs; case CEP_SCALE_GK1: return tt06::P_gK1;
        case CEP_SCALE_GBNA: return tt06::P_gbna; case CEP_SCALE_GBCA: return tt06::P_gbca;
        case CEP_SCALE_GPCA: return tt06::P_gpCa; case CEP_SCALE_GPK: return tt06::P_gpK;
        default: return -1;
      }
    case CEP_MODEL_TT2004:
      switch (g) {
        case CEP_SCALE_GNA: return tt04::P_gNa; case CEP_SCALE_GTO: return tt04::P_gto;
        case CEP_SCALE_GCAL: return tt04::P_gCaL; case CEP_SCALE_GKR: return tt04::P_gKr;
        case CEP_SCALE_GKS: return tt04::P_gKs; case CEP_SCALE_GK1: return tt04::P_gK1;
        case CEP_SCALE_GBNA: return tt04::P_gbna; case CEP_SCALE_GBCA: return tt04::P_gbca;
        case CEP_SCALE_GPCA: return tt04::P_gpCa; case CEP_SCALE_GPK: return tt04::P_gpK;
        default: return -1;
      }
    default: return -1;
  }
}

int cep_batch_scale(cep_batch_t b, int conductance, const double *factor) {
  if (!b || !factor) return fail(CEP_ERR_ARG, "null argument");
  if (!b->initialized) return fail(CEP_ERR_STATE, "cep_batch_init must come first");
  if (conductance < 0 || conductance >= CEP_SCALE_COUNT)
    return fail(CEP_ERR_ARG, "conductance %d is not a CEP_SCALE_* value", conductance);
  const int pidx = scale_param_index(b->model, conductance);
  if (pidx < 0) return fail(CEP_ERR_UNSUPPORTED, "model %d has no scalable parameter for conductance %d", b->model,
                            conductance);
  for (int i = 0; i < b->n; ++i)
    if (!std::isfinite(factor[i]) || factor[i] < 0.0)
      return fail(CEP_ERR_ARG, "factor[%d] = %g is not a finite non-negative value", i, factor[i]);
  double *d_f = nullptr;
  CEP_CUDA(cudaMallocAsync((void **)&d_f, sizeof(double) * b->n, b->stream));
  CEP_CUDA(cudaMemcpyAsync(d_f, factor, sizeof(double) * b->n, cudaMemcpyHostToDevice, b->stream));
  cep::scale_kernel<<<(b->n + kBlock - 1) / kBlock, kBlock, 0, b->stream>>>(b->params, b->ld, b->n, pidx, d_f);
  CEP_CUDA(cudaGetLastError());
  CEP_CUDA(cudaFreeAsync(d_f, b->stream));
  CEP_CUDA(cudaStreamSynchronize(b->stream));
  return CEP_OK;
}

static int conductance_row(cep_batch_t b, int conductance, int *pidx) {
  if (!b->initialized) return fail(CEP_ERR_STATE, "cep_batch_init must come first");
  if (conductance < 0 || conductance >= CEP_SCALE_COUNT)
    return fail(CEP_ERR_ARG, "conductance %d is not a CEP_SCALE_* value", conductance);
  *pidx = scale_param_index(b->model, conductance);
  if (*pidx < 0) return fail(CEP_ERR_UNSUPPORTED, "model %d has no parameter for conductance %d", b->model, conductance);
  return CEP_OK;
}

int cep_batch_get_conductance(cep_batch_t b, int conductance, double *values) {
  if (!b || !values) return fail(CEP_ERR_ARG, "null argument");
  int pidx = 0;
  const int rc = conductance_row(b, conductance, &pidx);
  if (rc) return rc;
  CEP_CUDA(cudaMemcpyAsync(values, b->params + (size_t)pidx * b->ld, sizeof(double) * b->n, cudaMemcpyDeviceToHost,
                           b->stream));
  CEP_CUDA(cudaStreamSynchronize(b->stream));
  return CEP_OK;
}

int cep_batch_set_conductance(cep_batch_t b, int conductance, const double *values) {
  if (!b || !values) return fail(CEP_ERR_ARG, "null argument");
  int pidx = 0;
  const int rc = conductance_row(b, conductance, &pidx);
  if (rc) return rc;
  for (int i = 0; i < b->n; ++i)
    if (!std::isfinite(values[i]) || values[i] < 0.0)
      return fail(CEP_ERR_ARG, "values[%d] = %g is not a finite non-negative value", i, values[i]);
  CEP_CUDA(cudaMemcpyAsync(b->params + (size_t)pidx * b->ld, values, sizeof(double) * b->n, cudaMemcpyHostToDevice,
                           b->stream));
  CEP_CUDA(cudaStreamSynchronize(b->stream));
  return CEP_OK;
}

// Largest dt (ms) at which the mixed path's slow gates may take the 4-term
// series of 1 - e^{-a}, a = dt/tau (cep_device.cuh rush_larsen): the series
// error a^5/120 stays below FP32 rounding while a <= 0.1. The slow gates'
// smallest time constants: ORd / CiPA-ORd 0.5 ms, ToR-ORd about 0.1 ms (j
// and jp near +50 mV), ten Tusscher 2 ms (fCass, fCa).
static double mixed_dt_max(int model) {
  switch (model) {
    case CEP_MODEL_ORD2011:
    case CEP_MODEL_CIPA2017: return 0.05;
    case CEP_MODEL_TOMEK2019: return 0.01;
    default: return 0.2;
  }
}
static int check_mixed_dt(cep_batch_t b, double dt) {
  if (b->precision == CEP_PREC_MIXED && dt > mixed_dt_max(b->model))
    return fail(CEP_ERR_UNSUPPORTED,
                "mixed precision of model %d is validated for dt <= %g ms (dt = %g): use FP64 or a smaller dt",
                b->model, mixed_dt_max(b->model), dt);
  return CEP_OK;
}

int cep_batch_set_protocol(cep_batch_t b, double dt, int n_pace, int first_pace, double dt_write,
                           double qnet_vm_threshold) {
  if (!b) return fail(CEP_ERR_ARG, "null batch");
  if (!b->initialized) return fail(CEP_ERR_STATE, "cep_batch_init must come first");
  if (!(dt > 0) || !(dt_write > 0) || n_pace <= 0 || first_pace >= n_pace)
    return fail(CEP_ERR_ARG, "bad protocol (dt=%g n_pace=%d first_pace=%d dt_write=%g)", dt, n_pace, first_pace, dt_write);
  if (int rc_dt = check_mixed_dt(b, dt)) return rc_dt;
  const ModelInfo *mi = model_info(b->model);
  b->dt = dt; b->n_pace = n_pace; b->first_pace = first_pace; b->dt_write = dt_write;
  b->qnet_thr = qnet_vm_threshold;
  // per-instance loop bounds from each instance's BCL, computed as the
  // reference computes them (cipa_drug_bench.cpp:136,188,240)
  std::vector<double> bcl(b->n);
  if (int rc_c = copy_sync(bcl.data(), b->params + (size_t)mi->p_bcl * b->ld, sizeof(double) * b->n,
                          cudaMemcpyDeviceToHost, b->stream))
    return rc_c;
  std::vector<int> sc((size_t)4 * b->ld, 0);
  const int print_freq = (int)((1. / dt) * dt_write);
  int max_per_beat = 1;
  for (int i = 0; i < b->n; ++i) {
    sc[i] = (int)((n_pace * bcl[i]) / dt);
    sc[b->ld + i] = (int)(bcl[i] / dt);
    sc[2 * b->ld + i] = print_freq;
    sc[3 * b->ld + i] = first_pace;
    const int per_beat = print_freq > 0 ? sc[b->ld + i] / print_freq + 2 : 2;
    if (per_beat > max_per_beat) max_per_beat = per_beat;
  }
  if (int rc_c = copy_sync(b->sched, sc.data(), sc.size() * sizeof(int), cudaMemcpyHostToDevice, b->stream))
    return rc_c;
  if (first_pace >= 0) {
    if (!b->bmf) {
      int rc;
      if ((rc = dev_alloc(b, &b->bmf, (size_t)bm::kNumF * b->ld)) || (rc = dev_alloc(b, &b->bmi, (size_t)bm::kNumI * b->ld)))
        return rc;
    }
    if (max_per_beat > b->ca_cap) {
      int rc;
      b->ca_cap = max_per_beat;
      if ((rc = dev_alloc(b, &b->ca_t, (size_t)b->ca_cap * b->ld)) || (rc = dev_alloc(b, &b->ca_v, (size_t)b->ca_cap * b->ld)))
        return rc;
    }
  }
  b->has_protocol = true;
  RunArgs a = make_args(b, 0);
  int rc = mi->reset(b, a, 0, b->n);
  if (rc) return rc;
  CEP_CUDA(cudaStreamSynchronize(b->stream));
  return CEP_OK;
}

int cep_batch_run(cep_batch_t b, long n_steps) {
  if (!b) return fail(CEP_ERR_ARG, "null batch");
  if (!b->initialized) return fail(CEP_ERR_STATE, "cep_batch_init must come first");
  if (n_steps < 0 || n_steps > 0x3fffffff) return fail(CEP_ERR_ARG, "n_steps out of range");
  if (n_steps == 0) return CEP_OK;
  RunArgs a = make_args(b, n_steps);
  if (!b->has_protocol) a.bm_on = 0;
  return model_info(b->model)->run(b, a);
}

int cep_batch_run_to_end(cep_batch_t b, long steps_per_launch) {
  if (!b) return fail(CEP_ERR_ARG, "null batch");
  if (!b->has_protocol) return fail(CEP_ERR_STATE, "cep_batch_set_protocol must come first");
  if (steps_per_launch <= 0) steps_per_launch = 20000;
  std::vector<int> st(b->n);
  for (;;) {
    int rc = cep_batch_run(b, steps_per_launch);
    if (rc) return rc;
    CEP_CUDA(cudaMemcpyAsync(st.data(), b->status, sizeof(int) * b->n, cudaMemcpyDeviceToHost, b->stream));
    CEP_CUDA(cudaStreamSynchronize(b->stream));
    bool running = false;
    for (int v : st) running |= (v == CEP_INST_RUNNING);
    if (!running) break;
  }
  return CEP_OK;
}

int cep_batch_set_states(cep_batch_t b, const double *states, int layout) {
  if (!b || !states) return fail(CEP_ERR_ARG, "null argument");
  if (layout == CEP_LAYOUT_SOA) {
    CEP_CUDA(cudaMemcpy2DAsync(b->states, sizeof(double) * b->ld, states, sizeof(double) * b->n,
                               sizeof(double) * b->n, b->ns, cudaMemcpyHostToDevice, b->stream));
  } else if (layout == CEP_LAYOUT_AOS) {
    std::vector<double> soa((size_t)b->ns * b->n);
    for (int i = 0; i < b->n; ++i)
      for (int k = 0; k < b->ns; ++k) soa[(size_t)k * b->n + i] = states[(size_t)i * b->ns + k];
    CEP_CUDA(cudaMemcpy2DAsync(b->states, sizeof(double) * b->ld, soa.data(), sizeof(double) * b->n,
                               sizeof(double) * b->n, b->ns, cudaMemcpyHostToDevice, b->stream));
    CEP_CUDA(cudaStreamSynchronize(b->stream));
  } else {
    return fail(CEP_ERR_ARG, "bad layout %d", layout);
  }
  CEP_CUDA(cudaStreamSynchronize(b->stream));
  return CEP_OK;
}

int cep_batch_get_states(cep_batch_t b, double *states, int layout) {
  if (!b || !states) return fail(CEP_ERR_ARG, "null argument");
  if (layout == CEP_LAYOUT_SOA) {
    CEP_CUDA(cudaMemcpy2DAsync(states, sizeof(double) * b->n, b->states, sizeof(double) * b->ld,
                               sizeof(double) * b->n, b->ns, cudaMemcpyDeviceToHost, b->stream));
    CEP_CUDA(cudaStreamSynchronize(b->stream));
  } else if (layout == CEP_LAYOUT_AOS) {
    std::vector<double> soa((size_t)b->ns * b->n);
    CEP_CUDA(cudaMemcpy2DAsync(soa.data(), sizeof(double) * b->n, b->states, sizeof(double) * b->ld,
                               sizeof(double) * b->n, b->ns, cudaMemcpyDeviceToHost, b->stream));
    CEP_CUDA(cudaStreamSynchronize(b->stream));
    for (int i = 0; i < b->n; ++i)
      for (int k = 0; k < b->ns; ++k) states[(size_t)i * b->ns + k] = soa[(size_t)k * b->n + i];
  } else {
    return fail(CEP_ERR_ARG, "bad layout %d", layout);
  }
  return CEP_OK;
}

int cep_batch_device_states(cep_batch_t b, void **dev_ptr, long *ld) {
  if (!b || !dev_ptr) return fail(CEP_ERR_ARG, "null argument");
  *dev_ptr = b->states;
  if (ld) *ld = (long)b->ld;
  return CEP_OK;
}

int cep_batch_get_biomarkers(cep_batch_t b, cep_biomarkers_t *out) {
  if (!b || !out) return fail(CEP_ERR_ARG, "null argument");
  if (!b->bmf) return fail(CEP_ERR_STATE, "biomarkers are off (set_protocol with first_pace >= 0)");
  cep_biomarkers_t *d = nullptr;
  CEP_CUDA(cudaMallocAsync((void **)&d, sizeof(cep_biomarkers_t) * b->n, b->stream));
  bm::View v{b->bmf, b->bmi, b->ca_t, b->ca_v, b->ca_cap, b->ld};
  collect_bm_kernel<<<(b->n + kBlock - 1) / kBlock, kBlock, 0, b->stream>>>(v, b->status, 0, b->n, d);
  CEP_CUDA(cudaGetLastError());
  CEP_CUDA(cudaMemcpyAsync(out, d, sizeof(cep_biomarkers_t) * b->n, cudaMemcpyDeviceToHost, b->stream));
  CEP_CUDA(cudaFreeAsync(d, b->stream));
  CEP_CUDA(cudaStreamSynchronize(b->stream));
  return CEP_OK;
}

int cep_batch_get_status(cep_batch_t b, int32_t *status) {
  if (!b || !status) return fail(CEP_ERR_ARG, "null argument");
  CEP_CUDA(cudaMemcpyAsync(status, b->status, sizeof(int) * b->n, cudaMemcpyDeviceToHost, b->stream));
  CEP_CUDA(cudaStreamSynchronize(b->stream));
  return CEP_OK;
}

// ------------------------------------------------------ instance ranges
namespace {
int check_range(cep_batch_t b, int first, int count) {
  if (!b) return fail(CEP_ERR_ARG, "null batch");
  if (first < 0 || count <= 0 || (int64_t)first + count > b->n)
    return fail(CEP_ERR_ARG, "range [%d, %d) outside the batch of %d", first, first + count, b->n);
  return CEP_OK;
}
__global__ void fill_status_kernel(int *status, int64_t first, int count, int value) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < count) status[first + k] = value;
}
}  // namespace

int cep_batch_reserve_biomarkers(cep_batch_t b, int max_samples_per_beat, double dt, double dt_write,
                                 double qnet_vm_threshold) {
  if (!b) return fail(CEP_ERR_ARG, "null batch");
  if (!b->initialized) return fail(CEP_ERR_STATE, "cep_batch_init must come first");
  if (max_samples_per_beat < 1 || !(dt > 0) || !(dt_write > 0)) return fail(CEP_ERR_ARG, "bad reservation");
  if (int rc_dt = check_mixed_dt(b, dt)) return rc_dt;
  int rc;
  if (!b->bmf && ((rc = dev_alloc(b, &b->bmf, (size_t)bm::kNumF * b->ld)) ||
                  (rc = dev_alloc(b, &b->bmi, (size_t)bm::kNumI * b->ld))))
    return rc;
  if (max_samples_per_beat + 2 > b->ca_cap) {
    b->ca_cap = max_samples_per_beat + 2;
    if ((rc = dev_alloc(b, &b->ca_t, (size_t)b->ca_cap * b->ld)) || (rc = dev_alloc(b, &b->ca_v, (size_t)b->ca_cap * b->ld)))
      return rc;
  }
  b->dt = dt;
  b->dt_write = dt_write;
  b->qnet_thr = qnet_vm_threshold;
  b->first_pace = 0;  // biomarkers possible; each instance's own first pace decides
  b->has_protocol = true;
  // every slot starts released
  fill_status_kernel<<<(b->n + 255) / 256, 256, 0, b->stream>>>(b->status, 0, b->n, CEP_INST_IDLE);
  CEP_CUDA(cudaGetLastError());
  CEP_CUDA(cudaStreamSynchronize(b->stream));
  return CEP_OK;
}

int cep_batch_init_range(cep_batch_t b, int first, int count, const double *celltype, const double *conc,
                         const double *hill, int hill_stride, unsigned flags) {
  int rc = check_range(b, first, count);
  if (rc) return rc;
  if (hill && hill_stride < 14) return fail(CEP_ERR_ARG, "hill_stride must be >= 14 (got %d)", hill_stride);
  if ((flags & CEP_FLAG_NEO_ORD) && b->model != CEP_MODEL_ORD2011)
    return fail(CEP_ERR_UNSUPPORTED, "CEP_FLAG_NEO_ORD selects a build of ORd 2011 only");
  if ((flags & CEP_FLAG_NEO_ORD) && (flags & CEP_FLAG_QUIRKS))
    return fail(CEP_ERR_ARG, "CEP_FLAG_NEO_ORD and CEP_FLAG_QUIRKS name two different builds");
  if (conc)
    for (int k = 0; k < count; ++k)
      if (!(conc[k] >= 0.0) || !std::isfinite(conc[k]))
        return fail(CEP_ERR_ARG, "conc[%d] = %g is not a finite non-negative value", k, conc[k]);
  if (hill)
    for (int k = 0; k < count; ++k)
      for (int j = 0; j < 14; ++j)
        if (!std::isfinite(hill[(size_t)k * hill_stride + j]) || hill[(size_t)k * hill_stride + j] < 0.0)
          return fail(CEP_ERR_ARG, "hill[%d][%d] is not a finite non-negative value", k, j);
  const size_t bytes_h = hill ? (size_t)count * hill_stride * sizeof(double) : 0;
  double *d = nullptr;
  CEP_CUDA(cudaMallocAsync((void **)&d, sizeof(double) * count * 2 + bytes_h + 64, b->stream));
  double *d_ct = d, *d_conc = d + count, *d_hill = hill ? d + 2 * count : nullptr;
  std::vector<double> zeros;
  if (!celltype || !conc) zeros.assign(count, 0.0);
  CEP_CUDA(cudaMemcpyAsync(d_ct, celltype ? celltype : zeros.data(), sizeof(double) * count, cudaMemcpyHostToDevice, b->stream));
  CEP_CUDA(cudaMemcpyAsync(d_conc, conc ? conc : zeros.data(), sizeof(double) * count, cudaMemcpyHostToDevice, b->stream));
  if (hill) CEP_CUDA(cudaMemcpyAsync(d_hill, hill, bytes_h, cudaMemcpyHostToDevice, b->stream));
  rc = model_info(b->model)->init(b, first, count, d_ct, d_conc, d_hill, hill_stride, flags);
  CEP_CUDA(cudaFreeAsync(d, b->stream));
  CEP_CUDA(cudaStreamSynchronize(b->stream));
  if (!rc) b->initialized = true;
  return rc;
}

int cep_batch_set_pacing_range(cep_batch_t b, int first, int count, double bcl, double stim_start, double stim_dur,
                               double amp_scale) {
  int rc = check_range(b, first, count);
  if (rc) return rc;
  if (!(bcl > 0) || !std::isfinite(bcl)) return fail(CEP_ERR_ARG, "bcl must be positive");
  return model_info(b->model)->pacing(b, first, count, bcl, stim_start, stim_dur, amp_scale);
}

int cep_batch_start_range(cep_batch_t b, int first, int count, int n_pace, int first_pace) {
  int rc = check_range(b, first, count);
  if (rc) return rc;
  if (!b->has_protocol) return fail(CEP_ERR_STATE, "cep_batch_reserve_biomarkers or cep_batch_set_protocol first");
  if (n_pace <= 0 || first_pace >= n_pace) return fail(CEP_ERR_ARG, "bad protocol (n_pace=%d first_pace=%d)", n_pace, first_pace);
  if (first_pace >= 0 && !b->bmf) return fail(CEP_ERR_STATE, "biomarkers were not reserved");
  const ModelInfo *mi = model_info(b->model);
  std::vector<double> bcl(count);
  CEP_CUDA(cudaMemcpyAsync(bcl.data(), b->params + (size_t)mi->p_bcl * b->ld + first, sizeof(double) * count,
                           cudaMemcpyDeviceToHost, b->stream));
  CEP_CUDA(cudaStreamSynchronize(b->stream));
  const double dt = b->dt;
  const int print_freq = (int)((1. / dt) * b->dt_write);
  std::vector<int> sc((size_t)4 * count);
  for (int k = 0; k < count; ++k) {
    sc[k] = (int)((n_pace * bcl[k]) / dt);
    sc[count + k] = (int)(bcl[k] / dt);
    sc[2 * count + k] = print_freq;
    sc[3 * count + k] = first_pace;
    const int per_beat = print_freq > 0 ? sc[count + k] / print_freq + 2 : 2;
    if (first_pace >= 0 && per_beat > b->ca_cap)
      return fail(CEP_ERR_ARG, "BCL %g needs %d Ca samples per beat, %d reserved", bcl[k], per_beat, b->ca_cap);
  }
  for (int r = 0; r < 4; ++r)
    CEP_CUDA(cudaMemcpyAsync(b->sched + (size_t)r * b->ld + first, sc.data() + (size_t)r * count, sizeof(int) * count,
                             cudaMemcpyHostToDevice, b->stream));
  RunArgs a = make_args(b, 0);
  a.bm_on = b->bmf ? 1 : 0;
  rc = mi->reset(b, a, first, count);
  if (rc) return rc;
  CEP_CUDA(cudaStreamSynchronize(b->stream));
  return CEP_OK;
}

int cep_batch_release_range(cep_batch_t b, int first, int count) {
  int rc = check_range(b, first, count);
  if (rc) return rc;
  fill_status_kernel<<<(count + 255) / 256, 256, 0, b->stream>>>(b->status, first, count, CEP_INST_IDLE);
  CEP_CUDA(cudaGetLastError());
  return CEP_OK;
}

int cep_batch_get_biomarkers_range(cep_batch_t b, int first, int count, cep_biomarkers_t *out) {
  int rc = check_range(b, first, count);
  if (rc) return rc;
  if (!out) return fail(CEP_ERR_ARG, "null argument");
  if (!b->bmf) return fail(CEP_ERR_STATE, "biomarkers are off");
  cep_biomarkers_t *d = nullptr;
  CEP_CUDA(cudaMallocAsync((void **)&d, sizeof(cep_biomarkers_t) * count, b->stream));
  bm::View v{b->bmf, b->bmi, b->ca_t, b->ca_v, b->ca_cap, b->ld};
  collect_bm_kernel<<<(count + kBlock - 1) / kBlock, kBlock, 0, b->stream>>>(v, b->status, first, count, d);
  CEP_CUDA(cudaGetLastError());
  CEP_CUDA(cudaMemcpyAsync(out, d, sizeof(cep_biomarkers_t) * count, cudaMemcpyDeviceToHost, b->stream));
  CEP_CUDA(cudaFreeAsync(d, b->stream));
  CEP_CUDA(cudaStreamSynchronize(b->stream));
  return CEP_OK;
}

int cep_batch_get_clock(cep_batch_t b, int i, long *step, double *t) {
  if (!b || i < 0 || i >= b->n) return fail(CEP_ERR_ARG, "bad instance index");
  int s = 0;
  double tt = 0;
  CEP_CUDA(cudaMemcpyAsync(&s, b->iout + i, sizeof(int), cudaMemcpyDeviceToHost, b->stream));
  CEP_CUDA(cudaMemcpyAsync(&tt, b->t + i, sizeof(double), cudaMemcpyDeviceToHost, b->stream));
  CEP_CUDA(cudaStreamSynchronize(b->stream));
  if (step) *step = s;
  if (t) *t = tt;
  return CEP_OK;
}

int cep_batch_sync(cep_batch_t b) {
  if (!b) return fail(CEP_ERR_ARG, "null batch");
  CEP_CUDA(cudaStreamSynchronize(b->stream));
  return CEP_OK;
}

int cep_batch_rates(cep_batch_t b, double t, double *dvdt, double *currents) {
  if (!b) return fail(CEP_ERR_ARG, "null batch");
  double *d = nullptr;
  CEP_CUDA(cudaMallocAsync((void **)&d, sizeof(double) * 8 * b->n, b->stream));
  int rc = model_info(b->model)->rates(b, t, d, d + b->n);
  if (rc) return rc;
  if (dvdt) CEP_CUDA(cudaMemcpyAsync(dvdt, d, sizeof(double) * b->n, cudaMemcpyDeviceToHost, b->stream));
  if (currents) CEP_CUDA(cudaMemcpyAsync(currents, d + b->n, sizeof(double) * 7 * b->n, cudaMemcpyDeviceToHost, b->stream));
  CEP_CUDA(cudaFreeAsync(d, b->stream));
  CEP_CUDA(cudaStreamSynchronize(b->stream));
  return CEP_OK;
}

int cep_batch_rates_all(cep_batch_t b, double t, double *rates) {
  if (!b || !rates) return fail(CEP_ERR_ARG, "null argument");
  if (!b->initialized) return fail(CEP_ERR_STATE, "cep_batch_init must come first");
  double *d = nullptr;
  const size_t bytes = sizeof(double) * (size_t)b->ns * b->n;
  CEP_CUDA(cudaMallocAsync((void **)&d, bytes, b->stream));
  int rc = model_info(b->model)->rates_all(b, t, d);
  if (!rc) CEP_CUDA(cudaMemcpyAsync(rates, d, bytes, cudaMemcpyDeviceToHost, b->stream));
  CEP_CUDA(cudaFreeAsync(d, b->stream));
  CEP_CUDA(cudaStreamSynchronize(b->stream));
  return rc;
}

}  // extern "C"

namespace {
// Device scratch of one blocking protocol call, released on every return.
struct Scratch {
  std::vector<void *> p;
  ~Scratch() {
    for (void *q : p) cudaFree(q);
  }
  template <class T>
  int get(T **out, size_t count) {
    void *q = nullptr;
    const cudaError_t e = cudaMalloc(&q, count * sizeof(T) + 256);
    if (e != cudaSuccess) {
      cudaGetLastError();
      return fail(CEP_ERR_OOM, "cudaMalloc(%zu bytes): %s", count * sizeof(T), cudaGetErrorString(e));
    }
    p.push_back(q);
    *out = static_cast<T *>(q);
    return CEP_OK;
  }
};
}  // namespace

extern "C" {

int cep_batch_restitution(cep_batch_t b, const double *bcl, int n_bcl, int n_pace, double dt,
                          long steps_per_launch, cep_apdr_record_t *out, int max_records, int *n_records) {
  if (!b) return fail(CEP_ERR_ARG, "null batch");
  if (!b->initialized) return fail(CEP_ERR_STATE, "cep_batch_init must come first");
  if (!bcl || n_bcl <= 0) return fail(CEP_ERR_ARG, "bcl list is empty");
  if (n_pace <= 0) return fail(CEP_ERR_ARG, "n_pace must be positive (got %d)", n_pace);
  if (!(dt > 0) || !std::isfinite(dt)) return fail(CEP_ERR_ARG, "dt must be positive");
  if (int rc_dt = check_mixed_dt(b, dt)) return rc_dt;
  if (max_records < 0 || (max_records > 0 && !out)) return fail(CEP_ERR_ARG, "bad record buffer");
  if (steps_per_launch <= 0) steps_per_launch = 20000;
  if (steps_per_launch > (1L << 30)) steps_per_launch = 1L << 30;
  std::vector<int> S(n_bcl), imax(n_bcl);
  int s_max = 1;
  long expected = 0;
  for (int k = 0; k < n_bcl; ++k) {
    if (!(bcl[k] > 0) || !std::isfinite(bcl[k])) return fail(CEP_ERR_ARG, "bcl[%d] must be positive", k);
    const double steps = bcl[k] / dt, total = (n_pace * bcl[k]) / dt;  // apdr_bench.cpp:128,169
    if (steps < 1 || total > 2.0e9) return fail(CEP_ERR_ARG, "bcl[%d]/dt out of range", k);
    S[k] = (int)steps;
    imax[k] = (int)total;
    if (S[k] > s_max) s_max = S[k];
    const long boundaries = ((long)imax[k] + 1) / S[k];
    if (boundaries > 2) expected += boundaries - 2;
  }
  if (n_records) *n_records = (int)expected;
  const ModelInfo *mi = model_info(b->model);
  Scratch sc;
  RestitArgs a;
  a.y = b->states; a.par = b->params; a.ld = b->ld; a.n = b->n; a.dt = dt;
  a.max_rec = max_records;
  int rc;
  if ((rc = sc.get(&a.rf, (size_t)kRF * b->ld))) return rc;
  if ((rc = sc.get(&a.ri, (size_t)kRI * b->ld))) return rc;
  if ((rc = sc.get(&a.trace, (size_t)s_max * b->ld))) return rc;
  a.rec = nullptr;
  if (max_records > 0 && (rc = sc.get(&a.rec, (size_t)max_records * b->n))) return rc;
  const int grid = (b->n + 127) / 128;
  restit_init_kernel<<<grid, 128, 0, b->stream>>>(a);
  CEP_CUDA(cudaGetLastError());
  for (int k = 0; k < n_bcl; ++k) {
    if ((rc = mi->pacing(b, 0, b->n, bcl[k], -1.0, -1.0, 1.0))) return rc;  // CONSTANTS[stim_period] = bcl (:105)
    a.bcl = bcl[k]; a.S = S[k]; a.imax = imax[k]; a.n_steps = (int)steps_per_launch;
    restit_segment_kernel<<<grid, 128, 0, b->stream>>>(a);
    CEP_CUDA(cudaGetLastError());
    const long total = (long)imax[k] + 1;
    for (long done = 0; done < total; done += steps_per_launch)
      if ((rc = mi->restit(b, a))) return rc;
  }
  std::vector<int> st(b->n);
  CEP_CUDA(cudaMemcpyAsync(st.data(), a.ri + (size_t)RI_status * b->ld, sizeof(int) * b->n, cudaMemcpyDeviceToHost,
                           b->stream));
  if (max_records > 0)
    CEP_CUDA(cudaMemcpyAsync(out, a.rec, sizeof(cep_apdr_record_t) * (size_t)max_records * b->n,
                             cudaMemcpyDeviceToHost, b->stream));
  CEP_CUDA(cudaStreamSynchronize(b->stream));
  for (int i = 0; i < b->n; ++i)
    if (st[i] != 0) return fail(CEP_ERR_NONFINITE, "instance %d turned non-finite during restitution", i);
  return CEP_OK;
}

int cep_batch_clamp(cep_batch_t b, const double *v, long n_samples, double t0, double dt, int current,
                    double *out) {
  if (!b) return fail(CEP_ERR_ARG, "null batch");
  if (!b->initialized) return fail(CEP_ERR_STATE, "cep_batch_init must come first");
  if (!v || !out || n_samples <= 0) return fail(CEP_ERR_ARG, "empty clamp trace");
  if (current < 0 || current > 6) return fail(CEP_ERR_ARG, "current index %d not in 0..6", current);
  if (!(dt > 0) || !std::isfinite(dt) || !std::isfinite(t0)) return fail(CEP_ERR_ARG, "bad t0/dt");
  if (int rc_dt = check_mixed_dt(b, dt)) return rc_dt;
  const int chunk = 2048;
  Scratch sc;
  ClampArgs a;
  a.y = b->states; a.par = b->params; a.ld = b->ld; a.n = b->n; a.current = current; a.dt = dt;
  double *dv = nullptr, *dout = nullptr;
  int rc;
  if ((rc = sc.get(&dv, chunk))) return rc;
  if ((rc = sc.get(&dout, (size_t)chunk * b->ld))) return rc;
  a.v = dv; a.out = dout;
  const ModelInfo *mi = model_info(b->model);
  double t = t0;
  for (long k0 = 0; k0 < n_samples; k0 += chunk) {
    const int m = (int)std::min<long>(chunk, n_samples - k0);
    CEP_CUDA(cudaMemcpyAsync(dv, v + k0, sizeof(double) * m, cudaMemcpyHostToDevice, b->stream));
    a.m = m;
    a.t0 = t;
    if ((rc = mi->clamp(b, a))) return rc;
    CEP_CUDA(cudaMemcpy2DAsync(out + (size_t)k0 * b->n, sizeof(double) * b->n, dout, sizeof(double) * b->ld,
                               sizeof(double) * b->n, m, cudaMemcpyDeviceToHost, b->stream));
    CEP_CUDA(cudaStreamSynchronize(b->stream));  // dv is reused by the next chunk
    for (int k = 0; k < m; ++k) t += dt;          // the kernel's clock, same additions
  }
  return CEP_OK;
}

int cep_batch_hrv(cep_batch_t b, const double *bcls, int n_bcl, double dt, double dt_write, int num_pace1,
                  long steps_per_launch, cep_hrv_record_t *out) {
  if (!b) return fail(CEP_ERR_ARG, "null batch");
  if (!b->initialized) return fail(CEP_ERR_STATE, "cep_batch_init must come first");
  if (b->model != CEP_MODEL_ORD2011) return fail(CEP_ERR_UNSUPPORTED, "the HRV bench drives ORd 2011 only");
  if (!bcls || n_bcl <= 0) return fail(CEP_ERR_ARG, "bcl list is empty");
  if (!out) return fail(CEP_ERR_ARG, "null record buffer");
  if (!(dt > 0) || !std::isfinite(dt) || !(dt_write > 0) || !std::isfinite(dt_write))
    return fail(CEP_ERR_ARG, "dt and dt_write must be positive");
  if (int rc_dt = check_mixed_dt(b, dt)) return rc_dt;
  const double pf = (1. / dt) * dt_write;  // hrv_bench.cpp:140
  if (!(pf >= 1.0) || pf > 2.0e9) return fail(CEP_ERR_ARG, "dt_write must be at least dt");
  const int print_freq = (int)pf;
  if (steps_per_launch <= 0) steps_per_launch = 20000;
  if (steps_per_launch > (1L << 30)) steps_per_launch = 1L << 30;
  // the last 250 paces are evaluated; fewer than 250 paces evaluate none
  // (the bench's size_t subtraction wraps, :244)
  const long first_eval = n_bcl >= 250 ? (long)n_bcl - 250 : (long)n_bcl + 1;
  std::vector<int> imax(n_bcl);
  long cap = 1;
  for (int k = 0; k < n_bcl; ++k) {
    if (!(bcls[k] > 0) || !std::isfinite(bcls[k])) return fail(CEP_ERR_ARG, "bcls[%d] must be positive", k);
    const double steps = bcls[k] / dt;
    if (steps > 2.0e9) return fail(CEP_ERR_ARG, "bcls[%d]/dt out of range", k);
    imax[k] = (int)steps;  // :223
    if (k >= first_eval) cap = std::max(cap, ((long)imax[k] + 1) / print_freq + 1);
  }
  Scratch sc;
  hrv::Args a{};
  a.y = b->states; a.par = b->params; a.ld = b->ld; a.n = b->n; a.dt = dt; a.print_freq = print_freq;
  a.max_evals = (int)steps_per_launch;
  a.n_eligible = n_bcl >= 250 ? 250 : 0;
  int rc;
  if ((rc = sc.get(&a.v.f, (size_t)hrv::kNumF * b->ld))) return rc;
  if ((rc = sc.get(&a.v.fi, (size_t)hrv::kNumI * b->ld))) return rc;
  if ((rc = sc.get(&a.v.ca_t, (size_t)cap * b->ld))) return rc;
  if ((rc = sc.get(&a.v.ca_v, (size_t)cap * b->ld))) return rc;
  a.v.ca_cap = (int)cap;
  a.v.ld = b->ld;
  cep_hrv_record_t *d_out = nullptr;
  if ((rc = sc.get(&d_out, (size_t)b->n))) return rc;
  const int grid = (b->n + 127) / 128, grid32 = (b->n + 31) / 32;
  const bool mixed = b->precision == CEP_PREC_MIXED;
  hrv::init_kernel<<<grid, 128, 0, b->stream>>>(a);
  CEP_CUDA(cudaGetLastError());
  double cumm = 0.0;  // CONSTANTS[cumm_BCL] (:330)
  for (int p = 0; p < n_bcl; ++p) {
    a.bcl = bcls[p]; a.cumm = cumm; a.imax = imax[p]; a.pace = p;
    a.last = p >= first_eval ? 1 : 0;
    a.replace = (p + 1 == num_pace1 - 249) ? 1 : 0;
    hrv::pace_begin_kernel<<<grid, 128, 0, b->stream>>>(a);
    // evaluations of a pace: one per call (imax + 1) plus at most two of a
    // sample alone (the rewound first call, the last call)
    const long evals = (long)imax[p] + 3;
    for (long done = 0; done < evals; done += steps_per_launch) {
      if (b->variant == CEP_KERNEL_ROLES) {
        if (mixed) hrv::calls_roles_kernel<Mixed><<<grid32, 128, 0, b->stream>>>(a);
        else hrv::calls_roles_kernel<F64><<<grid32, 128, 0, b->stream>>>(a);
      } else if (b->variant == CEP_KERNEL_PAIRS) {
        if (mixed) hrv::calls_pairs_kernel<Mixed><<<grid32, 64, 0, b->stream>>>(a);
        else hrv::calls_pairs_kernel<F64><<<grid32, 64, 0, b->stream>>>(a);
      } else {
        if (mixed) hrv::calls_kernel<Mixed><<<grid, 128, 0, b->stream>>>(a);
        else hrv::calls_kernel<F64><<<grid, 128, 0, b->stream>>>(a);
      }
    }
    hrv::pace_end_kernel<<<grid, 128, 0, b->stream>>>(a);
    CEP_CUDA(cudaGetLastError());
    cumm += bcls[p];
  }
  hrv::collect_kernel<<<grid, 128, 0, b->stream>>>(a, d_out);
  CEP_CUDA(cudaGetLastError());
  CEP_CUDA(cudaMemcpyAsync(out, d_out, sizeof(cep_hrv_record_t) * b->n, cudaMemcpyDeviceToHost, b->stream));
  CEP_CUDA(cudaStreamSynchronize(b->stream));
  return CEP_OK;
}

int cep_internal_batch_tissue_step(cep_batch_t b, const unsigned char *d_mask, double t, double bcl, double t_crt,
                                   double dur, int n_pace, const CepProto *proto, const unsigned char *d_mask2) {
  if (!b || !b->initialized) return fail(CEP_ERR_STATE, "tissue batch not initialised");
  TissueArgs a;
  a.y = b->states; a.par = b->params; a.ld = b->ld; a.n = b->n; a.t = t; a.dt = b->dt; a.mask = d_mask;
  a.proto = proto; a.mask2 = d_mask2;
  // the "square" mesh S1 window (heart.cpp:309-323)
  const int iia = (int)(t / bcl);
  a.stim_on = (iia < n_pace && t < (double)iia * bcl + dur + t_crt && t > (double)iia * bcl + t_crt) ? 1 : 0;
  return model_info(b->model)->tissue(b, a);
}

int cep_internal_batch_tissue_begin(cep_batch_t b, double dt) {
  if (!b || !b->initialized) return fail(CEP_ERR_STATE, "tissue batch not initialised");
  if (!(dt > 0)) return fail(CEP_ERR_ARG, "dt must be positive");
  if (int rc_dt = check_mixed_dt(b, dt)) return rc_dt;
  b->dt = dt; b->n_pace = 1; b->first_pace = -1; b->dt_write = 1.0; b->qnet_thr = -1e300;
  std::vector<int> sc((size_t)4 * b->ld, 0);
  for (int i = 0; i < b->n; ++i) {
    sc[i] = 0x7fffffff;             // no protocol end
    sc[b->ld + i] = 0x7fffffff;     // no beat boundary
    sc[3 * b->ld + i] = -1;         // biomarkers off
  }
  if (int rc_c = copy_sync(b->sched, sc.data(), sc.size() * sizeof(int), cudaMemcpyHostToDevice, b->stream))
    return rc_c;
  b->has_protocol = true;
  RunArgs a = make_args(b, 0);
  a.bm_on = 0;
  int rc = model_info(b->model)->reset(b, a, 0, b->n);
  if (rc) return rc;
  CEP_CUDA(cudaStreamSynchronize(b->stream));
  return CEP_OK;
}

double *cep_internal_batch_v(cep_batch_t b) { return b ? b->states : nullptr; }
void *cep_internal_batch_stream(cep_batch_t b) { return b ? (void *)b->stream : nullptr; }
int cep_internal_set_fail(int code, const char *msg) { return fail(code, "%s", msg); }

int cep_batch_step(cep_batch_t b, double t, double dt, int stim_mode) {
  if (!b) return fail(CEP_ERR_ARG, "null batch");
  if (!b->initialized) return fail(CEP_ERR_STATE, "cep_batch_init must come first");
  if (!(dt > 0) || !std::isfinite(t)) return fail(CEP_ERR_ARG, "bad t or dt");
  if (int rc_dt = check_mixed_dt(b, dt)) return rc_dt;
  if (stim_mode < -1 || stim_mode > 1) return fail(CEP_ERR_ARG, "stim_mode must be -1, 0 or 1");
  TissueArgs a;
  a.y = b->states; a.par = b->params; a.ld = b->ld; a.n = b->n; a.t = t; a.dt = dt; a.mask = nullptr;
  a.proto = nullptr; a.mask2 = nullptr;
  a.stim_on = stim_mode;
  return model_info(b->model)->tissue(b, a);
}

double cep_qinward(const cep_biomarkers_t *c, const cep_biomarkers_t *d) {
  if (!c || !d) return NAN;
  return ((d->inal_auc / c->inal_auc) + (d->ical_auc / c->ical_auc)) * 0.5;
}

}  // extern "C"
