// Heart-rate-variability pacing of ORd 2011 instances with the CiPA beat
// evaluation of the last 250 paces fused into the step loop.
//
// Follows CEPCell_NEO/modules/hrv_bench.cpp:146-343 on the fixed-step
// scheme (each CVode call to tnext is one step of the solver clock t_solver
// to tnext, none when tnext <= t_solver). Pace p lasts bcls[p]; its calls
// iout = 0 .. (int)(bcls[p]/dt) each end at tnext, after which the bench
// evaluates computeRates(tnext, y) (:233-245) and runs its beat machine on
// that sample. The clock carries over from pace to pace with tcurr and
// tnext rewound by one dt at the start of every pace after the first
// (:227-230), so the first call of a pace is of zero (or rounding-sized)
// length. The stimulus is on for stim_start + cumm_BCL <= t <
// stim_start + cumm_BCL + duration (Ohara_Rudy_2011.cpp:694-695), cumm_BCL
// being the sum of the earlier paces' BCLs (:330).
//
// The whole schedule (t_solver, tnext, tcurr, iout) is the same for every
// instance, so every thread replays it in the bench's own double
// arithmetic and the warps never diverge on it. The model is evaluated once
// per call: the rates the bench evaluates for the sample of call k are the
// rates at the start of the step of call k + 1 whenever both see the same
// stimulus flag (time enters computeRates only through the stimulus), so
// one evaluation serves both; the few calls where that fails (the rewound
// first call of a pace, the last call of a pace) get an evaluation of their
// own without an update.
#pragma once
#include "biomarkers.cuh"
#include "cep_device.cuh"
#include "model_ord.cuh"

namespace cep {
namespace hrv {

// SoA double fields [kNumF][ld]; the two beat records in bm::B_* order.
enum : int {
  F_T0 = 0,   // the beat being evaluated (temp_result)
  F_S0 = 15,  // the beat kept (cipa_result)
  F_qnet = 30, F_inal, F_ical,
  F_t_depol, F_r30, F_r50, F_r90,
  F_amp50, F_amp90, F_c50p, F_c90p, F_c50c, F_c90c, F_t_ca_peak,
  F_tsolver, F_tnext, F_tcurr,
  kNumF
};
// SoA int fields [kNumI][ld]
enum : int { I_iout = 0, I_pending, I_peak_found, I_eligible, I_n_ca, I_steepest, I_temp_bcl, I_best_bcl,
             I_status, kNumI };

struct Args {
  double *y;
  const double *par;
  int64_t ld;
  int n;
  bm::View v;       // f [kNumF][ld], fi [kNumI][ld], the Ca ring [ca_cap][ld]
  double dt;
  int print_freq;   // (int)((1. / dt) * dt_write), hrv_bench.cpp:140
  // the pace
  double bcl, cumm; // BCL and cumm_BCL of the pace
  int imax;         // (int)(BCL / dt), :223
  int pace;
  int last;         // pace >= n_bcl - 250: its beat is evaluated
  int replace;      // pace + 1 == num_pace1 - 249: the kept beat becomes this one (:336-338)
  int max_evals;    // model evaluations per launch
  int n_eligible;   // paces evaluated (the printed record's n_eligible)
};

__device__ __forceinline__ void reset_beat(const bm::View &v, int64_t i, int base, double vm, double ca) {
  bm::beat_init(v, i, base, vm, ca);  // cipa_t::init, CEPCell_NEO/modules/commons.hpp:88-109
}

// The per-instance schedule: the solver clock, the bench's tnext / tcurr /
// iout and whether the sample of the last call is still owed.
struct Clock {
  double tsolver, tnext, tcurr;
  int iout;
  bool pending;
};

// One evaluation: rates at (t, y) with stimulus flag `stim`; y advances by h
// when `upd`; when `sample`, the evaluation also gives the owed sample of
// call s_iout at time s_t (y before the update is that call's state).
struct Eval {
  double t, h, s_t;
  int stim, s_iout;
  bool upd, sample;
};

__device__ __forceinline__ int stim_flag(double t, double w0, double w1) { return (w0 <= t && t < w1) ? 1 : 0; }

// The next evaluation of the pace, advancing the clock past every call it
// completes; false once every call of the pace has been made and sampled.
__device__ __forceinline__ bool next_eval(Clock &k, int imax, double dt, double w0, double w1, Eval &e) {
  for (;;) {
    if (k.iout > imax) {  // the loop of the pace has ended (:231)
      if (!k.pending) return false;
      e = Eval{k.tcurr, 0.0, k.tcurr, stim_flag(k.tcurr, w0, w1), k.iout, false, true};
      k.pending = false;
      return true;
    }
    const double h = k.tnext - k.tsolver;
    if (h > 0) {
      const int su = stim_flag(k.tsolver, w0, w1);
      if (k.pending && stim_flag(k.tcurr, w0, w1) != su) {  // the owed sample needs its own rates
        e = Eval{k.tcurr, 0.0, k.tcurr, stim_flag(k.tcurr, w0, w1), k.iout, false, true};
        k.pending = false;
        return true;
      }
      e = Eval{k.tsolver, h, k.tcurr, su, k.iout, true, k.pending};
      k.tsolver = k.tnext;  // CVode reached tnext (:234)
      k.tcurr = k.tnext;    // :236
      ++k.iout;             // :239
      k.tnext += dt;        // :240
      k.pending = true;
      return true;
    }
    if (k.pending) {
      e = Eval{k.tcurr, 0.0, k.tcurr, stim_flag(k.tcurr, w0, w1), k.iout, false, true};
      k.pending = false;
      return true;
    }
    // a call that does not move the solver (tnext <= t_solver)
    k.tcurr = k.tnext;
    ++k.iout;
    k.tnext += dt;
    k.pending = true;
  }
}

// The beat machine's per-step fields, in registers for a launch.
struct Hot {
  double qnet, inal, ical, dvmdt_max, dvmdt_repol, ca_peak, r30, r50, r90;
  int peak_found, eligible, n_ca;
};

__device__ __forceinline__ void hot_load(const bm::View &v, int64_t i, Hot &h) {
  h.qnet = v.F(F_qnet, i); h.inal = v.F(F_inal, i); h.ical = v.F(F_ical, i);
  h.dvmdt_max = v.F(F_T0 + bm::B_dvmdt_max, i); h.dvmdt_repol = v.F(F_T0 + bm::B_dvmdt_repol, i);
  h.ca_peak = v.F(F_T0 + bm::B_ca_peak, i);
  h.r30 = v.F(F_r30, i); h.r50 = v.F(F_r50, i); h.r90 = v.F(F_r90, i);
  h.peak_found = v.I(I_peak_found, i); h.eligible = v.I(I_eligible, i); h.n_ca = v.I(I_n_ca, i);
}

__device__ __forceinline__ void hot_store(const bm::View &v, int64_t i, const Hot &h) {
  v.F(F_qnet, i) = h.qnet; v.F(F_inal, i) = h.inal; v.F(F_ical, i) = h.ical;
  v.F(F_T0 + bm::B_dvmdt_max, i) = h.dvmdt_max; v.F(F_T0 + bm::B_dvmdt_repol, i) = h.dvmdt_repol;
  v.F(F_T0 + bm::B_ca_peak, i) = h.ca_peak;
  v.F(F_r30, i) = h.r30; v.F(F_r50, i) = h.r50; v.F(F_r90, i) = h.r90;
  v.I(I_peak_found, i) = h.peak_found; v.I(I_eligible, i) = h.eligible; v.I(I_n_ca, i) = h.n_ca;
}

// One sample of an evaluated pace (:246-311): V, CAI, dVdt and the currents
// at sample iout (iout >= 1) of time tcurr.
__device__ __forceinline__ void sample(const bm::View &v, int64_t i, Hot &h, int iout, double tcurr, double dt,
                                       int print_freq, int peak_every, double repol_after, double V, double CAI,
                                       double dVdt, double INaL, double ICaL, double Ito, double IKr, double IKs,
                                       double IK1) {
  h.qnet += (INaL + ICaL + Ito + IKr + IKs + IK1) * dt;  // :247-249
  h.inal += INaL * dt;
  h.ical += ICaL * dt;
  if (iout % print_freq == 0 && h.n_ca < v.ca_cap) {  // the cai samples of the beat (:252-256)
    v.ca_t[(int64_t)h.n_ca * v.ld + i] = tcurr;
    v.ca_v[(int64_t)h.n_ca * v.ld + i] = CAI;
    ++h.n_ca;
  }
  if (h.dvmdt_max < dVdt) h.dvmdt_max = dVdt;  // :259
  if (iout % peak_every == 0 && !h.peak_found) {  // :262-275
    v.F(F_T0 + bm::B_vm_peak, i) = V;
    v.F(F_t_depol, i) = tcurr;
    if (V > 0.) {
      const double valley = v.F(F_T0 + bm::B_vm_valley, i);
      h.r30 = V - (0.3 * (V - valley));
      h.r50 = V - (0.5 * (V - valley));
      h.r90 = V - (0.9 * (V - valley));
      h.eligible = 1;
    }
    h.peak_found = 1;
  } else if (h.eligible && tcurr > repol_after) {  // :276-300
    if (h.r30 >= V && V >= h.r90 && h.dvmdt_repol < dVdt) h.dvmdt_repol = dVdt;
    if (h.r50 > V && V > h.r50 - 2) v.F(F_T0 + bm::B_apd50, i) = tcurr - v.F(F_t_depol, i);
    if (h.r90 > V && V > h.r90 - 2) v.F(F_T0 + bm::B_apd90, i) = tcurr - v.F(F_t_depol, i);
    if (h.ca_peak < CAI) {
      h.ca_peak = CAI;
      const double valley = v.F(F_T0 + bm::B_ca_valley, i);
      v.F(F_amp50, i) = CAI - (0.5 * (CAI - valley));
      v.F(F_amp90, i) = CAI - (0.9 * (CAI - valley));
      v.F(F_t_ca_peak, i) = tcurr;
    }
  }
}

__device__ __forceinline__ Clock clock_load(const bm::View &v, int64_t i) {
  return Clock{v.F(F_tsolver, i), v.F(F_tnext, i), v.F(F_tcurr, i), v.I(I_iout, i), v.I(I_pending, i) != 0};
}
__device__ __forceinline__ void clock_store(const bm::View &v, int64_t i, const Clock &k) {
  v.F(F_tsolver, i) = k.tsolver; v.F(F_tnext, i) = k.tnext; v.F(F_tcurr, i) = k.tcurr;
  v.I(I_iout, i) = k.iout; v.I(I_pending, i) = k.pending ? 1 : 0;
}

// Protocol start: both beat records from the initial state (:160-170).
__global__ void init_kernel(Args a) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  const double V = a.y[ord::V * a.ld + i], ca = a.y[ord::cai * a.ld + i];
  for (int k = 0; k < kNumF; ++k) a.v.F(k, i) = 0.0;
  for (int k = 0; k < kNumI; ++k) a.v.I(k, i) = 0;
  reset_beat(a.v, i, F_T0, V, ca);
  reset_beat(a.v, i, F_S0, V, ca);
  a.v.F(F_tnext, i) = a.dt;  // tnext = dt, tcurr = t_solver = 0 (:169)
  a.v.I(I_status, i) = CEP_INST_RUNNING;
}

// Start of a pace (:214-232).
__global__ void pace_begin_kernel(Args a) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n || a.v.I(I_status, i) != CEP_INST_RUNNING) return;
  const bm::View &v = a.v;
  v.F(F_t_ca_peak, i) = v.F(F_tcurr, i);  // t_ca_peak = tcurr before the rewind
  if (a.pace > 0) {
    v.F(F_tcurr, i) -= a.dt;
    v.F(F_tnext, i) -= a.dt;
  }
  if (a.last) {
    reset_beat(v, i, F_T0, a.y[ord::V * a.ld + i], a.y[ord::cai * a.ld + i]);
    v.I(I_n_ca, i) = 0;
  }
  v.F(F_qnet, i) = 0.; v.F(F_inal, i) = 0.; v.F(F_ical, i) = 0.;
  v.I(I_peak_found, i) = 0; v.I(I_eligible, i) = 0; v.I(I_iout, i) = 0; v.I(I_pending, i) = 0;
}

// End of a pace (:302-338): the Ca durations from the beat's samples (kept
// in time order, which is the order the bench sorts them into), the beat's
// record, the steepest-repolarisation choice and the one-off replacement.
__global__ void pace_end_kernel(Args a) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n || a.v.I(I_status, i) != CEP_INST_RUNNING) return;
  const bm::View &v = a.v;
  const int T = F_T0, S = F_S0;
  if (a.last) {
    const double t_ca_peak = v.F(F_t_ca_peak, i), amp50 = v.F(F_amp50, i), amp90 = v.F(F_amp90, i);
    double c50p = v.F(F_c50p, i), c90p = v.F(F_c90p, i), c50c = v.F(F_c50c, i), c90c = v.F(F_c90c, i);
    const int n = v.I(I_n_ca, i);
    for (int k = 0; k < n; ++k) {
      const double tk = v.ca_t[(int64_t)k * v.ld + i], ck = v.ca_v[(int64_t)k * v.ld + i];
      if (tk < t_ca_peak) {
        if (ck < amp50) c50p = tk;
        if (ck < amp90) c90p = tk;
      } else {
        if (ck > amp50) c50c = tk;
        if (ck > amp90) c90c = tk;
      }
    }
    v.F(F_c50p, i) = c50p; v.F(F_c90p, i) = c90p; v.F(F_c50c, i) = c50c; v.F(F_c90c, i) = c90c;
    v.F(T + bm::B_cad50, i) = c50c - c50p;
    v.F(T + bm::B_cad90, i) = c90c - c90p;
    v.F(T + bm::B_qnet, i) = v.F(F_qnet, i);
    v.F(T + bm::B_inal, i) = v.F(F_inal, i);
    v.F(T + bm::B_ical, i) = v.F(F_ical, i);
    v.F(T + bm::B_vm_dia, i) = a.y[ord::V * a.ld + i];
    v.F(T + bm::B_ca_dia, i) = a.y[ord::cai * a.ld + i];
    v.I(I_temp_bcl, i) = (int)a.bcl;
    if (v.F(T + bm::B_dvmdt_repol, i) > v.F(S + bm::B_dvmdt_repol, i)) {
      v.I(I_steepest, i) = a.pace;
      bm::beat_copy(v, i, S, T);
      v.I(I_best_bcl, i) = v.I(I_temp_bcl, i);
    }
  }
  if (a.replace) {
    bm::beat_copy(v, i, S, T);
    v.I(I_best_bcl, i) = v.I(I_temp_bcl, i);
  }
}

// The calls of one pace, one thread per instance, at most a.max_evals model
// evaluations per launch; the clock and the owed sample carry over to the
// next launch.
template <class P>
__global__ void __launch_bounds__(128) calls_kernel(Args a) {
  using G = typename P::G;
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n || a.v.I(I_status, i) != CEP_INST_RUNNING) return;
  const bm::View &v = a.v;
  Clock k = clock_load(v, i);
  if (k.iout > a.imax && !k.pending) return;
  ord::Y<G> y;
  ord::Par<G> q;
  ord::load(y, a.y, a.ld, i);
  ord::load_par(q, a.par, a.ld, i);
  const double stim_start = a.par[ord::P_stim_start * a.ld + i], dur = a.par[ord::P_duration * a.ld + i];
  const double w0 = stim_start + a.cumm, w1 = stim_start + a.cumm + dur;
  const double repol_after = a.cumm + (stim_start + 6.);
  int peak_every = (int)((stim_start + 6.) / a.dt);
  if (peak_every < 1) peak_every = 1;
  Hot h;
  if (a.last) hot_load(v, i, h);
  ord::Cur<G> c;
  int st = CEP_INST_RUNNING;
  Eval e;
  for (int n = 0; n < a.max_evals && next_eval(k, a.imax, a.dt, w0, w1, e); ++n) {
    const double V0 = y.V, cai0 = y.cai;
    ord::step<P>(y, q, e.t, e.h, e.stim, e.upd, c);
    if (a.last && e.sample)
      sample(v, i, h, e.s_iout, e.s_t, a.dt, a.print_freq, peak_every, repol_after, V0, cai0, (double)c.dVdt,
             (double)c.INaL, (double)c.ICaL, (double)c.Ito, (double)c.IKr, (double)c.IKs, (double)c.IK1);
    if (!isfinite(y.V)) {  // the bench only records it (:241-243); the instance stops here
      st = CEP_INST_NONFINITE;
      break;
    }
  }
  ord::store(y, a.y, a.ld, i);
  if (a.last) hot_store(v, i, h);
  clock_store(v, i, k);
  if (st != CEP_INST_RUNNING) v.I(I_status, i) = st;
}

// The warp-specialised form (as run_roles_kernel: 4 warps per 32 cells, one
// channel group each, the Parts summed through shared memory; warp 0 runs
// the beat machine). The schedule is uniform, so every lane of every warp
// takes the same evaluations.
template <class P, int R, int R2 = -1>
__device__ __forceinline__ void role_calls(const Args &a, typename P::G (*part)[4][8][32], int lane) {
  using G = typename P::G;
  const int64_t i = (int64_t)blockIdx.x * 32 + lane;
  const bool valid = i < a.n;
  const int64_t il = valid ? i : (int64_t)a.n - 1;
  const bm::View &v = a.v;
  bool alive = valid && v.I(I_status, il) == CEP_INST_RUNNING;
  Clock k = clock_load(v, il);
  alive = alive && !(k.iout > a.imax && !k.pending);
  if (!__syncthreads_or(alive)) return;
  ord::Y<G> y;
  ord::Par<G> q;
  ord::load(y, a.y, a.ld, il);
  ord::load_par(q, a.par, a.ld, il);
  const double stim_start = a.par[ord::P_stim_start * a.ld + il], dur = a.par[ord::P_duration * a.ld + il];
  const double w0 = stim_start + a.cumm, w1 = stim_start + a.cumm + dur;
  const double repol_after = a.cumm + (stim_start + 6.);
  int peak_every = (int)((stim_start + 6.) / a.dt);
  if (peak_every < 1) peak_every = 1;
  const bool bm_on = R == 0 && a.last;
  Hot h;
  if (bm_on) hot_load(v, il, h);
  ord::Cur<G> c;
  int st = CEP_INST_RUNNING;
  int buf = 0;
  Eval e;
  // every warp walks the same schedule for a lane; a lane whose instance has
  // stopped or finished the pace evaluates nothing but keeps meeting the
  // barrier until no lane of the block has work left
  bool more = alive;
  for (int n = 0; n < a.max_evals; ++n) {
    more = more && next_eval(k, a.imax, a.dt, w0, w1, e);
    if (!__syncthreads_or(more)) break;
    const bool active = alive && more;
    const double V0 = y.V, cai0 = y.cai;
    const auto ctx = ord::context<P>(y, q, e.t, e.stim);
    {
      ord::Part<G> p;
      ord::role<P, false, R>(y, q, ctx, e.h, active && e.upd, p);
#pragma unroll
      for (int f = 0; f < 8; ++f) {
        const int fld = ord::role_field<ord::kIK1InNa<P>>(R, f);
        if (fld >= 0) part[buf][R][f][lane] = p.f[fld];
      }
    }
    if constexpr (R2 >= 0) {
      ord::Part<G> p;
      ord::role<P, false, R2>(y, q, ctx, e.h, active && e.upd, p);
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
    ord::combine<P>(y, q, s, e.h, active && e.upd, c);
    if (bm_on && active && e.sample)
      sample(v, i, h, e.s_iout, e.s_t, a.dt, a.print_freq, peak_every, repol_after, V0, cai0, (double)c.dVdt,
             (double)c.INaL, (double)c.ICaL, (double)c.Ito, (double)c.IKr, (double)c.IKs, (double)c.IK1);
    if (active && !isfinite(y.V)) {
      st = CEP_INST_NONFINITE;
      alive = false;
    }
    buf ^= 1;
  }
  if (valid && (alive || st != CEP_INST_RUNNING)) {
    if (bm_on) hot_store(v, i, h);
    ord::store_role<false, ord::kIK1InNa<P>>(R, y, a.y, a.ld, i);
    if constexpr (R2 >= 0) ord::store_role<false, ord::kIK1InNa<P>>(R2, y, a.y, a.ld, i);
    if (R == 0) {
      clock_store(v, i, k);
      if (st != CEP_INST_RUNNING) v.I(I_status, i) = st;
    }
  }
}

template <class P>
__global__ void __launch_bounds__(128) calls_roles_kernel(Args a) {
  using G = typename P::G;
  __shared__ G part[2][4][8][32];
  const int lane = threadIdx.x & 31;
  switch (pick_role()) {
    case 0: role_calls<P, 0>(a, part, lane); break;
    case 1: role_calls<P, 1>(a, part, lane); break;
    case 2: role_calls<P, 2>(a, part, lane); break;
    default: role_calls<P, 3>(a, part, lane); break;
  }
}

template <class P>
__global__ void __launch_bounds__(64) calls_pairs_kernel(Args a) {
  using G = typename P::G;
  __shared__ G part[2][4][8][32];
  const int lane = threadIdx.x & 31;
  if ((threadIdx.x >> 5) == 0)
    role_calls<P, 0, 2>(a, part, lane);
  else
    role_calls<P, 1, 3>(a, part, lane);
}

// The printed record (:342-386): APD90 below APD50 reports the BCL.
__global__ void collect_kernel(Args a, cep_hrv_record_t *out) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  const bm::View &v = a.v;
  const int S = F_S0;
  cep_hrv_record_t o;
  cep_biomarkers_t &r = o.beat;
  const int bcl = v.I(I_best_bcl, i);
  r.qnet = v.F(S + bm::B_qnet, i) / 1000.0;
  r.inal_auc = v.F(S + bm::B_inal, i);
  r.ical_auc = v.F(S + bm::B_ical, i);
  r.dvmdt_repol = v.F(S + bm::B_dvmdt_repol, i);
  r.dvmdt_max = v.F(S + bm::B_dvmdt_max, i);
  r.vm_peak = v.F(S + bm::B_vm_peak, i);
  r.vm_valley = v.F(S + bm::B_vm_valley, i);
  r.vm_dia = v.F(S + bm::B_vm_dia, i);
  r.apd50 = v.F(S + bm::B_apd50, i);
  r.apd90 = v.F(S + bm::B_apd90, i);
  if (r.apd90 < r.apd50) r.apd90 = bcl;
  r.apd_tri = r.apd90 - r.apd50;
  r.ca_peak = v.F(S + bm::B_ca_peak, i);
  r.ca_valley = v.F(S + bm::B_ca_valley, i);
  r.ca_dia = v.F(S + bm::B_ca_dia, i);
  r.cad90 = v.F(S + bm::B_cad90, i);
  r.cad50 = v.F(S + bm::B_cad50, i);
  r.cad_tri = r.cad90 - r.cad50;
  r.steepest_pace = v.I(I_steepest, i);
  r.n_eligible = a.n_eligible;
  const int st = v.I(I_status, i);
  r.status = st == CEP_INST_RUNNING ? CEP_INST_DONE : st;
  r.reserved = 0;
  o.bcl = bcl;
  o.reserved = 0;
  out[i] = o;
}

}  // namespace hrv
}  // namespace cep
