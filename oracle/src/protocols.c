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
