// Per-instance CiPA biomarker state machine, fused into the ionic kernels.
//
// Follows CEPCell_NEO/modules/cipa_drug_bench.cpp:225-330 applied to the
// fixed-step trajectory: sample k (k = 1..imax) is the state after k steps
// at t_k with rates and currents evaluated at that state (the reference
// evaluates computeRates(tnext, y) after each CVode call, :215). The kernel
// evaluates rates at the start of step k, so the sample of step k is taken
// before the state update.
//
// The per-step modulo tests of the reference (iout % print_freq,
// iout % (BCL/dt), iout % ((BCL*pace + stim_start + 6)/dt)) are replaced by
// count-downs that fire on exactly the same steps. Traces never leave the
// device: cai samples of the current beat go to a per-instance ring in HBM
// and are reduced at the pace boundary.
#pragma once
#include "cep_device.cuh"

namespace cep {
namespace bm {

// SoA double fields [kNumF][ld]
enum : int {
  F_qnet = 0, F_inal, F_ical,          // running integrals of the current beat
  F_t_ca_peak, F_ca_amp50, F_ca_amp90,  // Ca bookkeeping of the current beat
  F_cad50_curr, F_cad50_prev, F_cad90_curr, F_cad90_prev,
  F_repol30, F_repol50, F_repol90, F_t_depol, F_peak_time,
  F_T0,                 // temp beat (15 fields) starts here
  F_S0 = F_T0 + 15,     // selected beat (15 fields)
  kNumF = F_S0 + 15
};
// SoA int fields [kNumI][ld]
enum : int { I_pace = 0, I_steepest, I_eligible, I_n_ca, I_n_elig, I_peak_step, I_next_peak, kNumI };
// beat record field offsets (same order as BeatRec)
enum : int {
  B_qnet = 0, B_inal, B_ical, B_dvmdt_repol, B_dvmdt_max, B_vm_peak, B_vm_valley, B_vm_dia, B_apd90,
  B_apd50, B_ca_peak, B_ca_valley, B_ca_dia, B_cad90, B_cad50
};

struct View {
  double *f;       // [kNumF][ld]
  int *fi;         // [kNumI][ld]
  double *ca_t;    // [ca_cap][ld]
  double *ca_v;    // [ca_cap][ld]
  int ca_cap;
  int64_t ld;
  __device__ __forceinline__ double &F(int k, int64_t i) const { return f[k * ld + i]; }
  __device__ __forceinline__ int &I(int k, int64_t i) const { return fi[k * ld + i]; }
};

// Per-instance protocol (host-computed, exactly as the reference computes
// its loop bounds: cipa_drug_bench.cpp:136,188,240).
struct Sched {
  int imax;           // (int)((n_pace * BCL) / dt)
  int steps_per_bcl;  // (int)(BCL / dt)
  int print_freq;     // (int)((1. / dt) * dt_write)
  int first_pace;     // first evaluated pace; < 0: biomarkers off
};

__device__ __forceinline__ void beat_init(const View &v, int64_t i, int base, double vm, double ca) {
  // cipa_t::init, CEPCell_NEO/modules/commons.hpp:88-109
  v.F(base + B_qnet, i) = 0.; v.F(base + B_inal, i) = 0.; v.F(base + B_ical, i) = 0.;
  v.F(base + B_dvmdt_repol, i) = -999; v.F(base + B_dvmdt_max, i) = -999;
  v.F(base + B_vm_peak, i) = -999; v.F(base + B_vm_valley, i) = vm; v.F(base + B_vm_dia, i) = -999;
  v.F(base + B_apd90, i) = 0.; v.F(base + B_apd50, i) = 0.; v.F(base + B_ca_peak, i) = -999;
  v.F(base + B_ca_valley, i) = ca; v.F(base + B_ca_dia, i) = -999; v.F(base + B_cad90, i) = 0.;
  v.F(base + B_cad50, i) = 0.;
}

__device__ __forceinline__ void beat_copy(const View &v, int64_t i, int dst, int src) {
#pragma unroll
  for (int k = 0; k < 15; ++k) v.F(dst + k, i) = v.F(src + k, i);
}

// (int)(((BCL*pace)+(stim_start+6.)) / dt): the step of the Vm-peak sample
// of pace `pace` (cipa_drug_bench.cpp:302).
__device__ __forceinline__ int peak_step(double bcl, int pace, double stim_start, double dt) {
  return (int)(((bcl * pace) + (stim_start + 6.)) / dt);
}
// Count-down for "iout % x == 0" tests: the number of sample calls, counting
// the first one, until the next multiple of x. A launch that starts at iout0
// makes its first sample call at max(iout0, 1) (sample 0 is the initial
// state, which the reference never evaluates).
__device__ __forceinline__ int countdown(int iout0, int x) {
  if (x <= 0) return 0x7fffffff;
  const int first = iout0 < 1 ? 1 : iout0;
  return (x - first % x) % x + 1;
}
__device__ __forceinline__ int next_multiple(int iout, int x) {
  if (x <= 0) return 0x7fffffff;
  const int r = iout % x;
  return r == 0 ? iout : iout + (x - r);
}

// Reset at protocol start (state = initial state of the instance).
__device__ __forceinline__ void reset(const View &v, int64_t i, double vm0, double ca0, double bcl,
                                      double stim_start, double dt) {
  for (int k = 0; k < kNumF; ++k) v.F(k, i) = 0.0;
  beat_init(v, i, F_T0, vm0, ca0);
  beat_init(v, i, F_S0, vm0, ca0);
  v.F(F_t_depol, i) = bcl * 0 + stim_start;
  v.F(F_peak_time, i) = (bcl * 0) + (stim_start + 6.);
  v.I(I_pace, i) = 0; v.I(I_steepest, i) = 0; v.I(I_eligible, i) = 0; v.I(I_n_ca, i) = 0;
  v.I(I_n_elig, i) = 0;
  const int ps = peak_step(bcl, 0, stim_start, dt);
  v.I(I_peak_step, i) = ps;
  v.I(I_next_peak, i) = next_multiple(1, ps);
}

// The fields the state machine touches on every step, held in registers for
// the length of a launch: loaded before the step loop (hot_load), written
// back after it (hot_store) and around the once-per-beat pace boundary,
// which works on the global record. Everything else stays in global memory.
struct Hot {
  double qnet, inal, ical;                    // running integrals of the beat
  double dvmdt_max, dvmdt_repol, ca_peak;     // of the temp beat record
  double peak_time, r30, r50, r90;            // Vm-peak time, repolarisation levels
  int pace, next_peak, eligible;
};

__device__ __forceinline__ void hot_load(const View &v, int64_t i, Hot &h) {
  h.qnet = v.F(F_qnet, i); h.inal = v.F(F_inal, i); h.ical = v.F(F_ical, i);
  h.dvmdt_max = v.F(F_T0 + B_dvmdt_max, i); h.dvmdt_repol = v.F(F_T0 + B_dvmdt_repol, i);
  h.ca_peak = v.F(F_T0 + B_ca_peak, i);
  h.peak_time = v.F(F_peak_time, i);
  h.r30 = v.F(F_repol30, i); h.r50 = v.F(F_repol50, i); h.r90 = v.F(F_repol90, i);
  h.pace = v.I(I_pace, i); h.next_peak = v.I(I_next_peak, i); h.eligible = v.I(I_eligible, i);
}

__device__ __forceinline__ void hot_store(const View &v, int64_t i, const Hot &h) {
  v.F(F_qnet, i) = h.qnet; v.F(F_inal, i) = h.inal; v.F(F_ical, i) = h.ical;
  v.F(F_T0 + B_dvmdt_max, i) = h.dvmdt_max; v.F(F_T0 + B_dvmdt_repol, i) = h.dvmdt_repol;
  v.F(F_T0 + B_ca_peak, i) = h.ca_peak;
  v.F(F_peak_time, i) = h.peak_time;
  v.F(F_repol30, i) = h.r30; v.F(F_repol50, i) = h.r50; v.F(F_repol90, i) = h.r90;
  v.I(I_pace, i) = h.pace; v.I(I_next_peak, i) = h.next_peak; v.I(I_eligible, i) = h.eligible;
}

// One sample (iout >= 1) of the state machine. V, CAI, dVdt and the six
// qNet currents are the values at sample iout; tcurr its time. h holds the
// hot fields (hot_load before the first sample of a launch).
__device__ __forceinline__ void sample(const View &v, int64_t i, const Sched &s, int iout, double tcurr,
                                       double dt, double bcl, double stim_start, double V, double CAI,
                                       double dVdt, double INaL, double ICaL, double Ito, double IKr,
                                       double IKs, double IK1, double qnet_thr, int &cnt_print,
                                       int &cnt_bcl, Hot &h) {
  // qnet and AUCs (:225-227)
  if (V > qnet_thr) {
    h.qnet += (INaL + ICaL + Ito + IKr + IKs + IK1) * dt;
    h.inal += INaL * dt;
    h.ical += ICaL * dt;
  }
  // cai samples of the evaluated beats (:230-235); cnt_print counts down to
  // the next multiple of print_freq
  if (--cnt_print == 0) {
    cnt_print = s.print_freq;
    if (h.pace >= s.first_pace) {
      const int n = v.I(I_n_ca, i);
      if (n < v.ca_cap) {
        v.ca_t[(int64_t)n * v.ld + i] = tcurr;
        v.ca_v[(int64_t)n * v.ld + i] = CAI;
        v.I(I_n_ca, i) = n + 1;
      }
    }
  }
  // pace boundary (:238-293), once per beat, on the global record
  if (--cnt_bcl == 0) {
    cnt_bcl = s.steps_per_bcl;
    hot_store(v, i, h);
    int pace = h.pace;
    if (v.I(I_eligible, i) && pace >= s.first_pace) {
      const double t_ca_peak = v.F(F_t_ca_peak, i), amp50 = v.F(F_ca_amp50, i), amp90 = v.F(F_ca_amp90, i);
      double c50c = v.F(F_cad50_curr, i), c50p = v.F(F_cad50_prev, i);
      double c90c = v.F(F_cad90_curr, i), c90p = v.F(F_cad90_prev, i);
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
      v.F(F_cad50_curr, i) = c50c; v.F(F_cad50_prev, i) = c50p;
      v.F(F_cad90_curr, i) = c90c; v.F(F_cad90_prev, i) = c90p;
      v.F(F_T0 + B_cad50, i) = c50c - c50p;
      v.F(F_T0 + B_cad90, i) = c90c - c90p;
      v.F(F_T0 + B_qnet, i) = v.F(F_qnet, i);
      v.F(F_T0 + B_inal, i) = v.F(F_inal, i);
      v.F(F_T0 + B_ical, i) = v.F(F_ical, i);
      v.F(F_T0 + B_vm_dia, i) = V;
      v.F(F_T0 + B_ca_dia, i) = CAI;
      v.I(I_n_elig, i) += 1;
      if (v.F(F_T0 + B_dvmdt_repol, i) > v.F(F_S0 + B_dvmdt_repol, i)) {
        v.I(I_steepest, i) = pace;
        beat_copy(v, i, F_S0, F_T0);
      }
    }
    pace += 1;
    v.I(I_pace, i) = pace;
    if (pace == s.first_pace + 1) {
      beat_copy(v, i, F_S0, F_T0);
      v.I(I_steepest, i) = pace - 1;
    }
    v.F(F_qnet, i) = 0.; v.F(F_inal, i) = 0.; v.F(F_ical, i) = 0.;
    if (pace >= s.first_pace) {
      beat_init(v, i, F_T0, V, CAI);
      v.I(I_n_ca, i) = 0;
      v.F(F_t_ca_peak, i) = tcurr;
      v.F(F_t_depol, i) = (bcl * pace) + stim_start;
      v.I(I_eligible, i) = 0;
    }
    const int ps = peak_step(bcl, pace, stim_start, dt);
    v.I(I_peak_step, i) = ps;
    v.I(I_next_peak, i) = next_multiple(iout, ps);
    v.F(F_peak_time, i) = (bcl * pace) + (stim_start + 6.);
    hot_load(v, i, h);
  }
  // last evaluated paces (:296-330)
  if (s.first_pace >= 0 && h.pace >= s.first_pace) {
    if (h.dvmdt_max < dVdt) h.dvmdt_max = dVdt;
    if (iout == h.next_peak) {
      h.next_peak = iout + v.I(I_peak_step, i);
      v.F(F_T0 + B_vm_peak, i) = V;
      if (V > 0.) {
        const double valley = v.F(F_T0 + B_vm_valley, i);
        h.r30 = V - (0.3 * (V - valley));
        h.r50 = V - (0.5 * (V - valley));
        h.r90 = V - (0.9 * (V - valley));
        h.eligible = 1;
      }
    } else if (h.eligible && tcurr > h.peak_time) {
      if (h.r30 >= V && V >= h.r90 && h.dvmdt_repol < dVdt) h.dvmdt_repol = dVdt;
      if (h.r50 > V && V > h.r50 - 2) v.F(F_T0 + B_apd50, i) = tcurr - v.F(F_t_depol, i);
      if (h.r90 > V && V > h.r90 - 2) v.F(F_T0 + B_apd90, i) = tcurr - v.F(F_t_depol, i);
      if (h.ca_peak < CAI) {
        h.ca_peak = CAI;
        const double valley = v.F(F_T0 + B_ca_valley, i);
        v.F(F_ca_amp50, i) = CAI - (0.5 * (CAI - valley));
        v.F(F_ca_amp90, i) = CAI - (0.9 * (CAI - valley));
        v.F(F_t_ca_peak, i) = tcurr;
      }
    }
  } else if (iout == h.next_peak) {
    h.next_peak = iout + v.I(I_peak_step, i);
  }
}

}  // namespace bm
}  // namespace cep
