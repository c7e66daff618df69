/*
 * TEST INFRASTRUCTURE ONLY. Model dispatch, the reference's fixed-step
 * driver loop, the CiPA biomarker state machine and a threaded batch runner
 * (the CPU baseline) for the CPU oracle.
 */
#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>
#include "cep_oracle.h"

/* per-model entry points (ord2011.c, cipa2017.c, tt2006.c, tt2004.c, tomek2019.c) */
int cepo_ord_init(cepo_cell *, double, double, const double *, int, int);
void cepo_ord_init_states(double *);
void cepo_ord_set_pacing(cepo_cell *, double, double, double, double);
void cepo_ord_step(const cepo_cell *, double, double, double *, cepo_currents *);
void cepo_ord_rates(const cepo_cell *, double, const double *, double *, cepo_currents *);

int cepo_cipa_init(cepo_cell *, double, double, const double *, int, int);
void cepo_cipa_init_states(const cepo_cell *, double *);
void cepo_cipa_set_pacing(cepo_cell *, double, double, double, double);
void cepo_cipa_step(const cepo_cell *, double, double, double *, cepo_currents *);
void cepo_cipa_rates(const cepo_cell *, double, const double *, double *, cepo_currents *);

int cepo_tt06_init(cepo_cell *, double, double, const double *, int, int);
void cepo_tt06_init_states(double *);
void cepo_tt06_set_pacing(cepo_cell *, double, double, double, double);
void cepo_tt06_step(const cepo_cell *, double, double, double *, cepo_currents *);
void cepo_tt06_rates(const cepo_cell *, double, const double *, double *, cepo_currents *);

int cepo_tt04_init(cepo_cell *, double, double, const double *, int, int);
void cepo_tt04_init_states(double *);
void cepo_tt04_set_pacing(cepo_cell *, double, double, double, double);
void cepo_tt04_step(const cepo_cell *, double, double, double *, cepo_currents *);
void cepo_tt04_rates(const cepo_cell *, double, const double *, double *, cepo_currents *);

int cepo_tomek_init(cepo_cell *, double, double, const double *, int, int);
void cepo_tomek_init_states(const cepo_cell *, double *);
void cepo_tomek_set_pacing(cepo_cell *, double, double, double, double);
void cepo_tomek_step(const cepo_cell *, double, double, double *, cepo_currents *);
void cepo_tomek_rates(const cepo_cell *, double, const double *, double *, cepo_currents *);

void cepo_ord_pacing(const cepo_cell *, double *, double *);
void cepo_cipa_pacing(const cepo_cell *, double *, double *);
void cepo_tt06_pacing(const cepo_cell *, double *, double *);
void cepo_tt04_pacing(const cepo_cell *, double *, double *);
void cepo_tomek_pacing(const cepo_cell *, double *, double *);

void cepo_pacing_of(const cepo_cell *c, double *bcl, double *stim_start) {
  switch (c->model) {
    case CEPO_ORD2011: cepo_ord_pacing(c, bcl, stim_start); break;
    case CEPO_CIPA2017: cepo_cipa_pacing(c, bcl, stim_start); break;
    case CEPO_TT2006: cepo_tt06_pacing(c, bcl, stim_start); break;
    case CEPO_TT2004: cepo_tt04_pacing(c, bcl, stim_start); break;
    case CEPO_TOMEK2019: cepo_tomek_pacing(c, bcl, stim_start); break;
  }
}

/* index of intracellular Ca in each model's STATES */
int cepo_cai_index(int model) {
  switch (model) {
    case CEPO_TT2006: return 3;
    case CEPO_TT2004: return 3;
    default: return 9;
  }
}

int cepo_n_states(int model) {
  switch (model) {
    case CEPO_ORD2011: return 41;
    case CEPO_CIPA2017: return 49;
    case CEPO_TT2006: return 19;
    case CEPO_TT2004: return 17;
    case CEPO_TOMEK2019: return 43;
  }
  return -1;
}

int cepo_init(cepo_cell *c, int model, double celltype, double conc, const double *hill, int n_hill,
              int is_dutta, int quirks) {
  double row[CEPO_MAX_HILL];
  memset(row, 0, sizeof(row));
  if (hill) {
    if (n_hill > CEPO_MAX_HILL) n_hill = CEPO_MAX_HILL;
    memcpy(row, hill, sizeof(double) * (size_t)n_hill);
  }
  memset(c, 0, sizeof(*c));
  c->model = model;
  c->quirks = quirks;
  switch (model) {
    case CEPO_ORD2011: return cepo_ord_init(c, celltype, conc, hill ? row : NULL, is_dutta, quirks);
    case CEPO_CIPA2017: return cepo_cipa_init(c, celltype, conc, row, is_dutta, quirks);
    case CEPO_TT2006: return cepo_tt06_init(c, celltype, conc, row, is_dutta, quirks);
    case CEPO_TT2004: return cepo_tt04_init(c, celltype, conc, row, is_dutta, quirks);
    case CEPO_TOMEK2019: return cepo_tomek_init(c, celltype, conc, row, is_dutta, quirks);
  }
  return -1;
}

void cepo_init_states(const cepo_cell *c, double *y) {
  switch (c->model) {
    case CEPO_ORD2011: cepo_ord_init_states(y); break;
    case CEPO_CIPA2017: cepo_cipa_init_states(c, y); break;
    case CEPO_TT2006: cepo_tt06_init_states(y); break;
    case CEPO_TT2004: cepo_tt04_init_states(y); break;
    case CEPO_TOMEK2019: cepo_tomek_init_states(c, y); break;
  }
}

void cepo_set_pacing(cepo_cell *c, double bcl, double stim_start, double stim_dur, double amp_scale) {
  switch (c->model) {
    case CEPO_ORD2011: cepo_ord_set_pacing(c, bcl, stim_start, stim_dur, amp_scale); break;
    case CEPO_CIPA2017: cepo_cipa_set_pacing(c, bcl, stim_start, stim_dur, amp_scale); break;
    case CEPO_TT2006: cepo_tt06_set_pacing(c, bcl, stim_start, stim_dur, amp_scale); break;
    case CEPO_TT2004: cepo_tt04_set_pacing(c, bcl, stim_start, stim_dur, amp_scale); break;
    case CEPO_TOMEK2019: cepo_tomek_set_pacing(c, bcl, stim_start, stim_dur, amp_scale); break;
  }
}

int cepo_scale(cepo_cell *c, int g, double f) {
  switch (c->model) {
    case CEPO_ORD2011: return cepo_ord_scale(c, g, f);
    case CEPO_CIPA2017: return cepo_cipa_scale(c, g, f);
    case CEPO_TT2006: return cepo_tt06_scale(c, g, f);
    case CEPO_TT2004: return cepo_tt04_scale(c, g, f);
    case CEPO_TOMEK2019: return cepo_tomek_scale(c, g, f);
  }
  return -1;
}

void cepo_step(const cepo_cell *c, double t, double dt, double *y, cepo_currents *cur) {
  switch (c->model) {
    case CEPO_ORD2011: cepo_ord_step(c, t, dt, y, cur); break;
    case CEPO_CIPA2017: cepo_cipa_step(c, t, dt, y, cur); break;
    case CEPO_TT2006: cepo_tt06_step(c, t, dt, y, cur); break;
    case CEPO_TT2004: cepo_tt04_step(c, t, dt, y, cur); break;
    case CEPO_TOMEK2019: cepo_tomek_step(c, t, dt, y, cur); break;
  }
}

void cepo_rates(const cepo_cell *c, double t, const double *y, double *dydt, cepo_currents *cur) {
  switch (c->model) {
    case CEPO_ORD2011: cepo_ord_rates(c, t, y, dydt, cur); break;
    case CEPO_CIPA2017: cepo_cipa_rates(c, t, y, dydt, cur); break;
    case CEPO_TT2006: cepo_tt06_rates(c, t, y, dydt, cur); break;
    case CEPO_TT2004: cepo_tt04_rates(c, t, y, dydt, cur); break;
    case CEPO_TOMEK2019: cepo_tomek_rates(c, t, y, dydt, cur); break;
  }
}

/* The reference's explicit loop, CEPCell_HACKATHON/modules/
 * cipa_drug_explicit_bench.cpp:119-127. */
void cepo_run(const cepo_cell *c, double *t, double dt, long n_steps, double *y, double *v_trace,
              long v_stride) {
  double tc = *t;
  long k = 0;
  for (long i = 0; i < n_steps; ++i) {
    cepo_step(c, tc, dt, y, NULL);
    tc += dt;
    if (v_trace && v_stride > 0 && ((i + 1) % v_stride) == 0) v_trace[k++] = y[0];
  }
  *t = tc;
}

static void beat_init(cepo_beat *b, double vm, double ca) {
  /* cipa_t::init, CEPCell_NEO/modules/commons.hpp:88-109 */
  b->qnet = 0.; b->inal_auc = 0.; b->ical_auc = 0.;
  b->dvmdt_repol = -999; b->dvmdt_max = -999; b->vm_peak = -999; b->vm_valley = vm;
  b->vm_dia = -999; b->apd90 = 0.; b->apd50 = 0.; b->ca_peak = -999; b->ca_valley = ca;
  b->ca_dia = -999; b->cad90 = 0.; b->cad50 = 0.;
}

/* Fixed-step form of the CiPA bench loop, CEPCell_NEO/modules/
 * cipa_drug_bench.cpp:199-330. Sample k (k = 1..imax) is the state after k
 * steps at tcurr = t_k, with rates and currents evaluated at that state, as
 * the reference evaluates computeRates(tnext, y) after each CVode call
 * (:215). The fixed-step trajectory is the explicit scheme of
 * cipa_drug_explicit_bench.cpp:119-127. Paces >= first_pace are evaluated
 * (the reference uses num_pace1-250 and gates the block on num_pace1>250,
 * :296; first_pace >= 0 replaces that gate). */
int cepo_run_biomarkers(const cepo_cell *c, double *y, double dt, int n_pace, int first_pace,
                        double dt_write, double qnet_vm_threshold, cepo_biomarkers *out,
                        double *v_trace, long v_stride, long v_cap) {
  const int ns = cepo_n_states(c->model);
  double BCL, stim_start;
  cepo_pacing_of(c, &BCL, &stim_start);
  const int print_freq = (int)((1. / dt) * dt_write);
  const int imax = (int)((n_pace * BCL) / dt);
  const int steps_per_bcl = (int)(BCL / dt);
  cepo_beat cipa, temp;
  double qnet = 0, inal_auc = 0, ical_auc = 0;
  double t_ca_peak = 0, ca_amp50 = 0, ca_amp90 = 0;
  double cad50_curr = 0, cad50_prev = 0, cad90_curr = 0, cad90_prev = 0;
  double vm_repol30 = 0, vm_repol50 = 0, vm_repol90 = 0;
  int pace = 0, steepest = 0, eligible = 0, n_elig = 0;
  double t_depol = BCL * pace + stim_start;
  /* cai samples of the current beat (at most one per print_freq steps) */
  const long cap = steps_per_bcl / (print_freq > 0 ? print_freq : 1) + 4;
  double *ca_t = (double *)malloc(sizeof(double) * (size_t)cap);
  double *ca_v = (double *)malloc(sizeof(double) * (size_t)cap);
  long n_ca = 0;
  long kv = 0;
  cepo_currents cur;
  double tcurr = 0.0;
  const int cai_idx = cepo_cai_index(c->model);
  beat_init(&cipa, y[0], y[cai_idx]);
  temp = cipa;
  int status = 0;
  for (int iout = 1; iout <= imax; ++iout) {
    cepo_step(c, tcurr, dt, y, NULL);
    tcurr += dt;
    cepo_rates(c, tcurr, y, NULL, &cur);
    if (!(y[0] == y[0]) || fabs(y[0]) > 1e6) { status = 1; break; }
    if (v_trace && v_stride > 0 && (iout % v_stride) == 0 && kv < v_cap) v_trace[kv++] = y[0];
    const double V_ = y[0], CAI = y[cai_idx];
    if (V_ > qnet_vm_threshold) {
      qnet += (cur.INaL + cur.ICaL + cur.Ito + cur.IKr + cur.IKs + cur.IK1) * dt;
      inal_auc += cur.INaL * dt;
      ical_auc += cur.ICaL * dt;
    }
    if (pace >= first_pace && iout % print_freq == 0 && n_ca < cap) {
      ca_t[n_ca] = tcurr;
      ca_v[n_ca] = CAI;
      n_ca++;
    }
    if (iout > 0 && iout % steps_per_bcl == 0) {
      if (eligible && pace >= first_pace) {
        for (long k = 0; k < n_ca; ++k) {
          if (ca_t[k] < t_ca_peak) {
            if (ca_v[k] < ca_amp50) cad50_prev = ca_t[k];
            if (ca_v[k] < ca_amp90) cad90_prev = ca_t[k];
          } else {
            if (ca_v[k] > ca_amp50) cad50_curr = ca_t[k];
            if (ca_v[k] > ca_amp90) cad90_curr = ca_t[k];
          }
        }
        temp.cad50 = cad50_curr - cad50_prev;
        temp.cad90 = cad90_curr - cad90_prev;
        temp.qnet = qnet;
        temp.inal_auc = inal_auc;
        temp.ical_auc = ical_auc;
        temp.vm_dia = V_;
        temp.ca_dia = CAI;
        n_elig++;
        if (temp.dvmdt_repol > cipa.dvmdt_repol) {
          steepest = pace;
          cipa = temp;
        }
      }
      pace++;
      if (pace == first_pace + 1) {
        cipa = temp;
        steepest = pace - 1;
      }
      qnet = inal_auc = ical_auc = 0.;
      if (pace >= first_pace) {
        beat_init(&temp, V_, CAI);
        n_ca = 0;
        t_ca_peak = tcurr;
        t_depol = (BCL * pace) + stim_start;
        eligible = 0;
      }
    }
    if (first_pace >= 0 && pace >= first_pace) {
      if (temp.dvmdt_max < cur.dVdt) temp.dvmdt_max = cur.dVdt;
      if (iout % (int)(((BCL * pace) + (stim_start + 6.)) / dt) == 0) {
        temp.vm_peak = V_;
        if (temp.vm_peak > 0.) {
          vm_repol30 = temp.vm_peak - (0.3 * (temp.vm_peak - temp.vm_valley));
          vm_repol50 = temp.vm_peak - (0.5 * (temp.vm_peak - temp.vm_valley));
          vm_repol90 = temp.vm_peak - (0.9 * (temp.vm_peak - temp.vm_valley));
          eligible = 1;
        }
      } else if (eligible && tcurr > (BCL * pace) + (stim_start + 6.)) {
        if (vm_repol30 >= V_ && V_ >= vm_repol90 && temp.dvmdt_repol < cur.dVdt) temp.dvmdt_repol = cur.dVdt;
        if (vm_repol50 > V_ && V_ > vm_repol50 - 2) temp.apd50 = tcurr - t_depol;
        if (vm_repol90 > V_ && V_ > vm_repol90 - 2) temp.apd90 = tcurr - t_depol;
        if (temp.ca_peak < CAI) {
          temp.ca_peak = CAI;
          ca_amp50 = temp.ca_peak - (0.5 * (temp.ca_peak - temp.ca_valley));
          ca_amp90 = temp.ca_peak - (0.9 * (temp.ca_peak - temp.ca_valley));
          t_ca_peak = tcurr;
        }
      }
    }
  }
  (void)ns;
  free(ca_t);
  free(ca_v);
  if (out) {
    out->result = cipa;
    out->steepest_pace = steepest;
    out->n_eligible = n_elig;
    out->qnet_last = cipa.qnet / 1000.0;
    out->status = status;
  }
  return status;
}

/* ------------------------------------------------------ threaded baseline */
typedef struct {
  int model, n_hill, is_dutta, quirks;
  const double *celltype, *conc, *hill;
  double bcl, dt;
  long n_steps;
  double *states_out;
  int lo, hi;
} batch_job;

static void *batch_worker(void *arg) {
  batch_job *b = (batch_job *)arg;
  const int ns = cepo_n_states(b->model);
  for (int i = b->lo; i < b->hi; ++i) {
    cepo_cell c;
    cepo_init(&c, b->model, b->celltype ? b->celltype[i] : 0.0, b->conc ? b->conc[i] : 0.0,
              b->hill ? b->hill + (size_t)i * (size_t)b->n_hill : NULL, b->n_hill, b->is_dutta,
              b->quirks);
    cepo_set_pacing(&c, b->bcl, 10.0, -1.0, 1.0);
    double y[CEPO_MAX_STATES];
    cepo_init_states(&c, y);
    double t = 0.0;
    cepo_run(&c, &t, b->dt, b->n_steps, y, NULL, 0);
    if (b->states_out) memcpy(b->states_out + (size_t)i * (size_t)ns, y, sizeof(double) * (size_t)ns);
  }
  return NULL;
}

int cepo_run_batch(int model, int n, const double *celltype, const double *conc, const double *hill,
                   int n_hill, int is_dutta, int quirks, double bcl, double dt, long n_steps,
                   double *states_out, int n_threads) {
  if (n_threads < 1) n_threads = 1;
  if (n_threads > n) n_threads = n;
  pthread_t th[256];
  batch_job jobs[256];
  if (n_threads > 256) n_threads = 256;
  for (int k = 0; k < n_threads; ++k) {
    batch_job *b = &jobs[k];
    b->model = model; b->n_hill = n_hill; b->is_dutta = is_dutta; b->quirks = quirks;
    b->celltype = celltype; b->conc = conc; b->hill = hill; b->bcl = bcl; b->dt = dt;
    b->n_steps = n_steps; b->states_out = states_out;
    b->lo = (int)((long)n * k / n_threads);
    b->hi = (int)((long)n * (k + 1) / n_threads);
    pthread_create(&th[k], NULL, batch_worker, b);
  }
  for (int k = 0; k < n_threads; ++k) pthread_join(th[k], NULL);
  return n_threads;
}
