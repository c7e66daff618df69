/* TEST INFRASTRUCTURE ONLY: CPU restatement of the reference's protocol
 * benches on the fixed-step scheme, the checker of the device protocols.
 *
 * cepo_restitution: dynamic (S1-S1) restitution of
 * CEPCell_NEO/modules/apdr_bench.cpp:103-232. The reference integrates with
 * CVODE; here every iout is one fixed step (cepo_step), t advanced by
 * t += dt from 0 in each BCL segment as tnext is (:111-112, :139). The
 * per-pace Vm record vm_data is a std::multimap keyed by time (:50, :146):
 * it is cleared at every pace boundary (:208) but not between BCL segments,
 * so the steps after a segment's last boundary stay in it during the next
 * segment's first pace. This restatement keeps exactly that (entries sorted
 * by time, insertion order among equal times, when the search runs). */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "cep_oracle.h"

void cepo_pacing_of(const cepo_cell *c, double *bcl, double *stim_start);

typedef struct {
  double t, v;
  long seq;
} vm_entry;

static int cmp_entry(const void *a, const void *b) {
  const vm_entry *x = (const vm_entry *)a, *y = (const vm_entry *)b;
  if (x->t < y->t) return -1;
  if (x->t > y->t) return 1;
  return (x->seq < y->seq) ? -1 : (x->seq > y->seq);
}

int cepo_restitution(const cepo_cell *c0, double *y, const double *bcls, int n_bcl, int n_pace, double dt,
                     cepo_apdr_record *out, int max_records, int *n_records) {
  cepo_cell c = *c0;
  double bcl0, stim_start;
  cepo_pacing_of(&c, &bcl0, &stim_start);
  long cap = 1024, n_data = 0, seq = 0;
  for (int s = 0; s < n_bcl; ++s) {
    const long steps = (long)(bcls[s] / dt) + 2;
    if (steps > cap) cap = steps;
  }
  cap = 2 * cap + 16; /* a pace plus the steps left over from the previous segment */
  vm_entry *data = (vm_entry *)malloc(sizeof(vm_entry) * (size_t)cap);
  vm_entry *sorted = (vm_entry *)malloc(sizeof(vm_entry) * (size_t)cap);
  if (!data || !sorted) {
    free(data);
    free(sorted);
    return -1;
  }
  int is_replaced = 0, all_pace = 0, n_rec = 0, recal = 0, status = 0;
  double vm_valley = y[0], vm_peak = y[0], vm_repol = 0.0;
  double t_depol = 0.0, t_repol = 0.0, apd90 = 0.0, t_peak = 0.0, t_di;
  for (int s = 0; s < n_bcl && !status; ++s) {
    const double bcl = bcls[s];
    cepo_set_pacing(&c, bcl, -1.0, -1.0, 1.0); /* CONSTANTS[stim_period] = bcl (:105) */
    double tcurr = 0.0;
    int pace = 0;
    long iout = 0;
    const long imax = (long)((n_pace * bcl) / dt); /* :128 */
    const long S = (long)(bcl / dt);                /* :169 */
    t_depol = 0;
    t_repol = 0;
    while (iout <= imax) { /* :131 */
      cepo_step(&c, tcurr, dt, y, NULL);
      iout++;
      tcurr += dt;
      const double V = y[0];
      if (!isfinite(V)) {
        status = 1;
        break;
      }
      if (n_data < cap) {
        data[n_data].t = tcurr;
        data[n_data].v = V;
        data[n_data].seq = seq++;
        n_data++;
      }
      const double lo = (bcl * pace) + stim_start;
      /* vm_peak in the window, vm_repol after it (:149-157) */
      if (lo + 4. < tcurr && tcurr < lo + 56.) {
        if (vm_peak < V) {
          vm_peak = V;
          t_peak = tcurr;
        }
      } else if (tcurr > lo + 56.) {
        vm_repol = vm_peak - (0.9 * (vm_peak - vm_valley));
      }
      /* repolarisation (:161-166) */
      if (tcurr > lo + 56. && vm_repol >= V && V > vm_repol - 2) {
        t_depol = lo;
        t_repol = tcurr;
        apd90 = t_repol - t_depol;
        is_replaced = 1;
      }
      /* pace boundary (:169-213) */
      if (iout % S == 0) {
        if (vm_peak < 0 || (vm_peak >= 0 && vm_peak < 10)) {
          is_replaced = 0;
          recal = 1;
          memcpy(sorted, data, sizeof(vm_entry) * (size_t)n_data);
          qsort(sorted, (size_t)n_data, sizeof(vm_entry), cmp_entry);
          for (long k = 0; k < n_data; ++k) {
            if (vm_peak < sorted[k].v) {
              vm_peak = sorted[k].v;
              vm_repol = vm_peak - (0.9 * (vm_peak - vm_valley));
              t_peak = sorted[k].t;
            }
          }
          for (long k = 0; k < n_data; ++k) {
            if (sorted[k].t > t_peak && vm_repol >= sorted[k].v && sorted[k].v > vm_repol - 1) {
              t_depol = lo;
              t_repol = sorted[k].t;
              apd90 = t_repol - t_depol;
              is_replaced = 1;
            }
          }
        }
        if (!is_replaced) {
          t_depol = lo;
          t_repol = tcurr;
          apd90 = t_repol - t_depol;
        }
        vm_valley = V;
        vm_peak = -999;
        vm_repol = 0;
        pace++;
        all_pace++;
        is_replaced = 0;
        n_data = 0;
        if (pace > 2) {
          t_di = (tcurr + stim_start) - t_repol;
          if (n_rec < max_records) {
            cepo_apdr_record *r = &out[n_rec];
            r->pace = all_pace;
            r->recal = recal;
            r->bcl = bcl;
            r->apd90 = apd90;
            r->di = t_di;
            r->t = tcurr;
          }
          n_rec++;
        }
        recal = 0;
      }
    }
  }
  free(data);
  free(sorted);
  if (n_records) *n_records = n_rec;
  return status;
}

/* Voltage-clamp replay (CEPPatch/benchpatch.cpp:83-100): V is set to v[k]
 * before step k (rhs_fn sets y[V] = glob_vm, :20), the step runs from
 * t0 + k*dt (t += dt), and out[k] receives channel current `current`
 * (0 INa .. 6 IK1, the cepo_currents order) of that step. */
void cepo_clamp(const cepo_cell *c, double *y, const double *v, long n_samples, double t0, double dt,
                int current, double *out) {
  double t = t0;
  for (long k = 0; k < n_samples; ++k) {
    cepo_currents cur;
    y[0] = v[k];
    cepo_step(c, t, dt, y, &cur);
    const double vals[7] = {cur.INa, cur.INaL, cur.Ito, cur.ICaL, cur.IKr, cur.IKs, cur.IK1};
    out[k] = (current >= 0 && current < 7) ? vals[current] : 0.0;
    t += dt;
  }
}

/* ------------------------------------------------------------- HRV pacing
 * CEPCell_NEO/modules/hrv_bench.cpp:146-343 for one cell of ORd 2011 (the
 * CEPCell_NEO build, quirks 2) at one concentration:
 *  - one pace per entry of bcls: CONSTANTS[BCL] = bcls[k] (:176), the
 *    integrals reset (:180), iout = 0 .. imax = (int)(BCL / dt) inclusive
 *    (:181, :191), the stimulus window at cumm_BCL + stim_start
 *    (Ohara_Rudy_2011.cpp:695), cumm_BCL += BCL after the pace (:331);
 *  - every pace after the first rewinds tcurr and tnext by dt (:185-188):
 *    its first call asks CVODE for the time it has already reached, which
 *    returns the state unchanged; here that call is no step at all, and,
 *    like every call, it still adds the currents times dt to the integrals;
 *  - computeRates(tnext) after each call (:196) gives the currents and
 *    RATES[V] of the sample; the last 250 entries are evaluated (:216-265,
 *    with the bench's unsigned arithmetic: fewer than 250 entries evaluate
 *    none), the steepest repolarisation kept (:268-299); the record of pace
 *    num_pace1 - 249 replaces the selection once (:334-336, the bench
 *    tests p_param->num_pace1, not the number of entries);
 *  - afterwards an APD90 below the APD50 becomes the beat's BCL (:352).
 * The bench leaves t_depol, the repolarisation levels, the Ca amplitudes,
 * the CaD crossing times and the steepest pace uninitialised until first
 * set; here they start at 0. The Ca samples of a pace are sorted by time
 * (a std::multimap in the bench, :209). */
typedef struct {
  double t, c;
  long seq;
} ca_entry;

static int cmp_ca(const void *a, const void *b) {
  const ca_entry *x = (const ca_entry *)a, *y = (const ca_entry *)b;
  if (x->t < y->t) return -1;
  if (x->t > y->t) return 1;
  return (x->seq < y->seq) ? -1 : (x->seq > y->seq);
}

static void beat_reset(cepo_beat *b, double vm, double ca) {  /* cipa_t::init, commons.hpp:88-108 */
  memset(b, 0, sizeof(*b));
  b->dvmdt_repol = -999; b->dvmdt_max = -999; b->vm_peak = -999; b->vm_valley = vm; b->vm_dia = -999;
  b->ca_peak = -999; b->ca_valley = ca; b->ca_dia = -999;
}

int cepo_hrv_run(const cepo_cell *c0, double *y, const double *bcls, int n_bcl, double dt, double dt_write,
                 int num_pace1, cepo_hrv_record *rec) {
  cepo_cell c = *c0;
  c.tissue_stim = 2;
  double bcl0, stim_start;
  cepo_pacing_of(&c, &bcl0, &stim_start);
  const int print_freq = (int)((1. / dt) * dt_write);
  const int peak_every = (int)((stim_start + 6.) / dt);
  const long first_eval = n_bcl >= 250 ? n_bcl - 250 : (long)n_bcl + 1;  /* size_t wrap: none evaluated */
  double tcurr = 0.0, tnext = dt, t_solver = 0.0, cumm = 0.0;
  cepo_beat best, temp;
  beat_reset(&best, y[0], y[9]);
  beat_reset(&temp, y[0], y[9]);
  int best_bcl = 0, temp_bcl = 0, steepest = 0;
  double t_depol = 0, r30 = 0, r50 = 0, r90 = 0, amp50 = 0, amp90 = 0;
  double c50p = 0, c90p = 0, c50c = 0, c90c = 0;
  long cap = 4096, n_ca = 0;
  ca_entry *ca = malloc(sizeof(ca_entry) * cap);
  int status = 0;
  for (int pace = 0; pace < n_bcl; ++pace) {
    const double bcl = bcls[pace];
    cepo_set_pacing(&c, bcl, -1.0, -1.0, 1.0);
    cepo_ord_set_cumm(&c, cumm);
    double qnet = 0, inal = 0, ical = 0;
    const int imax = (int)(bcl / dt);
    int peak_found = 0, eligible = 0;
    double t_ca_peak = tcurr;
    if (pace > 0) {
      tcurr -= dt;
      tnext -= dt;
    }
    const int last = pace >= first_eval;
    if (last) {
      beat_reset(&temp, y[0], y[9]);
      n_ca = 0;
    }
    for (int iout = 0; iout <= imax;) {
      const double h = tnext - t_solver;
      if (h > 0) {
        cepo_step(&c, t_solver, h, y, NULL);
        t_solver = tnext;
      }
      tcurr = tnext;
      double dydt[CEPO_MAX_STATES];
      cepo_currents cur;
      cepo_rates(&c, tnext, y, dydt, &cur);
      ++iout;
      tnext += dt;
      if (!isfinite(y[0])) status = 1;
      qnet += (cur.INaL + cur.ICaL + cur.Ito + cur.IKr + cur.IKs + cur.IK1) * dt;
      inal += cur.INaL * dt;
      ical += cur.ICaL * dt;
      if (!last) continue;
      if (iout % print_freq == 0) {
        if (n_ca == cap) ca = realloc(ca, sizeof(ca_entry) * (cap *= 2));
        ca[n_ca].t = tcurr; ca[n_ca].c = y[9]; ca[n_ca].seq = n_ca; ++n_ca;
      }
      const double V = y[0], dV = dydt[0];
      if (temp.dvmdt_max < dV) temp.dvmdt_max = dV;
      if (iout % peak_every == 0 && !peak_found) {
        temp.vm_peak = V;
        t_depol = tcurr;
        if (temp.vm_peak > 0.) {
          r30 = temp.vm_peak - (0.3 * (temp.vm_peak - temp.vm_valley));
          r50 = temp.vm_peak - (0.5 * (temp.vm_peak - temp.vm_valley));
          r90 = temp.vm_peak - (0.9 * (temp.vm_peak - temp.vm_valley));
          eligible = 1;
        }
        peak_found = 1;
      } else if (eligible && tcurr > cumm + (stim_start + 6.)) {
        if (r30 >= V && V >= r90 && temp.dvmdt_repol < dV) temp.dvmdt_repol = dV;
        if (r50 > V && V > r50 - 2) temp.apd50 = tcurr - t_depol;
        if (r90 > V && V > r90 - 2) temp.apd90 = tcurr - t_depol;
        if (temp.ca_peak < y[9]) {
          temp.ca_peak = y[9];
          amp50 = temp.ca_peak - (0.5 * (temp.ca_peak - temp.ca_valley));
          amp90 = temp.ca_peak - (0.9 * (temp.ca_peak - temp.ca_valley));
          t_ca_peak = tcurr;
        }
      }
    }
    if (last) {
      qsort(ca, (size_t)n_ca, sizeof(ca_entry), cmp_ca);
      for (long k = 0; k < n_ca; ++k) {
        if (ca[k].t < t_ca_peak) {
          if (ca[k].c < amp50) c50p = ca[k].t;
          if (ca[k].c < amp90) c90p = ca[k].t;
        } else {
          if (ca[k].c > amp50) c50c = ca[k].t;
          if (ca[k].c > amp90) c90c = ca[k].t;
        }
      }
      temp.cad50 = c50c - c50p;
      temp.cad90 = c90c - c90p;
      temp.qnet = qnet;
      temp.inal_auc = inal;
      temp.ical_auc = ical;
      temp.vm_dia = y[0];
      temp.ca_dia = y[9];
      temp_bcl = (int)bcl;
      if (temp.dvmdt_repol > best.dvmdt_repol) {
        steepest = pace;
        best = temp;
        best_bcl = temp_bcl;
      }
    }
    cumm += bcl;
    if (pace + 1 == num_pace1 - 249) {
      best = temp;
      best_bcl = temp_bcl;
    }
  }
  free(ca);
  if (best.apd90 < best.apd50) best.apd90 = best_bcl;
  rec->beat = best;
  rec->bcl = best_bcl;
  rec->steepest_pace = steepest;
  return status;
}
