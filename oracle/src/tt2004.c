/*
 * TEST INFRASTRUCTURE ONLY. CPU restatement of the ten Tusscher - Noble -
 * Noble - Panfilov 2004 model as CEPCell_NEO/cellmodels/
 * tentusscher_noble_noble_panfilov_2004_b.cpp implements it with every
 * channel macro of its header defined (tentusscher_noble_noble_panfilov_
 * 2004_b.hpp:7-21): initConsts (:185-359), the Hill hook initConsts(type,
 * conc, hill) (:361-377), computeRates (:379-635, the standard INa branch,
 * glob_var::A1656D_mode = 0) and solveAnalytical (:637-658: Rush-Larsen for
 * ten gates, forward Euler for V, K_i, Na_i, Ca_i, Ca_SR, fCa and g), in the
 * reference's evaluation order (pinned bit for bit against the reference
 * compiled from its own sources).
 *
 * Quirk: the reference never assigns CONSTANTS[gmma] (the NaCa voltage
 * partition), so its value is whatever the heap held; in the reference
 * build here it was a denormal (6.9e-310) that acts exactly as 0. With
 * quirks the oracle uses 0; without, the published 0.35.
 */
#include <math.h>
#include <string.h>
#include "cep_oracle.h"

typedef struct {
  double R, T, F, Cm, V_c, stim_start, stim_period, stim_duration, stim_amplitude, P_kna, K_o, Na_o, Ca_o;
  double g_K1, g_Kr, g_Ks, g_Na, g_bna, g_CaL, g_bca, g_to, P_NaK, K_mk, K_mNa, K_NaCa, K_sat, alpha, gmma;
  double Km_Ca, Km_Nai, g_pCa, K_pCa, g_pK, tau_g, a_rel, b_rel, c_rel, K_up, V_leak, Vmax_up, Buf_c, K_buf_c;
  double Buf_sr, K_buf_sr, V_sr, tau_fCa;
} tt04_p;

enum { V = 0, K_i, Na_i, Ca_i, Xr1, Xr2, Xs, m, h, j, d, f, fCa, s, r, Ca_SR, g, TT04_NS };

static double hb(double D, double ic50, double hh) {
  return (ic50 > 10E-14 && hh > 10E-14) ? pow(1. + pow(D / ic50, hh), -1) : 1.;
}

int cepo_tt04_init(cepo_cell *c, double celltype, double conc, const double *hill, int is_dutta, int quirks) {
  (void)celltype; (void)is_dutta;
  tt04_p *q = (tt04_p *)c->p;
  memset(c->p, 0, sizeof(c->p));
  q->stim_start = 10; q->stim_period = 1000; q->stim_duration = 1; q->stim_amplitude = 52;
  q->R = 8314.472; q->T = 310; q->F = 96485.3415; q->Cm = 0.185; q->V_c = 0.016404;
  q->Na_o = 140; q->Ca_o = 2; q->K_o = 5.4; q->Buf_c = 0.15; q->K_buf_c = 0.001; q->Km_Nai = 87.5;
  q->Km_Ca = 1.38; q->K_NaCa = 1000; q->K_sat = 0.1; q->alpha = 2.5; q->K_mk = 1; q->K_mNa = 40;
  q->P_NaK = 1.362; q->g_bca = 0.000592; q->g_bna = 0.00029; q->g_CaL = 0.000175; q->tau_fCa = 2.00000;
  q->V_leak = 8e-5; q->Buf_sr = 10; q->K_buf_sr = 0.3; q->V_sr = 0.001094; q->a_rel = 0.016464;
  q->b_rel = 0.25; q->c_rel = 0.008232; q->tau_g = 2; q->Vmax_up = 0.000425; q->K_up = 0.00025;
  q->g_K1 = 5.405; q->g_Kr = 0.096; q->g_Ks = 0.245; q->P_kna = 0.03; q->g_Na = 14.838; q->g_pK = 0.0146;
  q->g_pCa = 0.825; q->K_pCa = 0.0005; q->g_to = 0.294;
  q->gmma = quirks ? 0.0 : 0.35;
  if (hill) {
    q->g_CaL *= hb(conc, hill[0], hill[1]);
    q->g_K1 *= hb(conc, hill[2], hill[3]);
    q->g_Ks *= hb(conc, hill[4], hill[5]);
    q->g_Na *= hb(conc, hill[6], hill[7]);
    q->g_to *= hb(conc, hill[10], hill[11]);
    q->g_Kr *= hb(conc, hill[12], hill[13]);
  }
  return 0;
}

/* The 2004_a build (tentusscher_noble_noble_panfilov_2004_a.cpp:265): the
 * same model with g_Ks = 0.062 (M cell) instead of 0.245; the Hill factor of
 * initConsts(type, conc, hill) applies on top, as in init. */
void cepo_tt04_mcell(cepo_cell *c, double conc, const double *hill) {
  tt04_p *q = (tt04_p *)c->p;
  q->g_Ks = 0.062;
  if (hill) q->g_Ks *= hb(conc, hill[4], hill[5]);
}

void cepo_tt04_init_states(double *y) {
  y[V] = -86.2; y[K_i] = 138.3; y[Na_i] = 11.6; y[Ca_i] = 0.0002; y[Xr1] = 0; y[Xr2] = 1; y[Xs] = 0;
  y[m] = 0; y[h] = 0.75; y[j] = 0.75; y[d] = 0; y[f] = 1; y[fCa] = 1; y[s] = 1; y[r] = 0; y[Ca_SR] = 0.2;
  y[g] = 1;
}

void cepo_tt04_set_pacing(cepo_cell *c, double bcl, double stim_start, double stim_dur, double amp_scale) {
  tt04_p *q = (tt04_p *)c->p;
  q->stim_period = bcl;
  if (stim_start >= 0) q->stim_start = stim_start;
  if (stim_dur >= 0) q->stim_duration = stim_dur;
  q->stim_amplitude *= amp_scale;
}

void cepo_tt04_pacing(const cepo_cell *c, double *bcl, double *stim_start) {
  const tt04_p *q = (const tt04_p *)c->p;
  *bcl = q->stim_period;
  *stim_start = q->stim_start;
}

typedef struct {
  double inf[10], tau[10];  /* RL pairs in solveAnalytical's order */
} tt04_alg;

/* computeRates, :379-635 */
static void tt04_compute(const cepo_cell *c, double TIME, const double *S, double *R_, tt04_alg *al,
                         cepo_currents *cur) {
  const tt04_p *q = (const tt04_p *)c->p;
  const double v = S[V];
  double i_Stim;
  if (c->tissue_stim) {
    i_Stim = c->is_s1 ? -q->stim_amplitude : 0.0;
  } else {
    i_Stim = (TIME - floor(TIME / q->stim_period) * q->stim_period >= q->stim_start &&
                      TIME - floor(TIME / q->stim_period) * q->stim_period <= q->stim_start + q->stim_duration
                  ? -q->stim_amplitude
                  : 0.000000);
  }
  const double RT = q->R * q->T;
  const double i_NaCa = (q->K_NaCa * (exp((q->gmma * v * q->F) / RT) * pow(S[Na_i], 3.00000) * q->Ca_o -
                                      exp(((q->gmma - 1.00000) * v * q->F) / RT) * pow(q->Na_o, 3.00000) * S[Ca_i] * q->alpha)) /
                        ((pow(q->Km_Nai, 3.00000) + pow(q->Na_o, 3.00000)) * (q->Km_Ca + q->Ca_o) *
                         (1.00000 + q->K_sat * exp(((q->gmma - 1.00000) * v * q->F) / RT)));
  const double Ca_i_bufc = 1.00000 / (1.00000 + (q->Buf_c * q->K_buf_c) / pow(S[Ca_i] + q->K_buf_c, 2.00000));
  const double i_NaK = (((q->P_NaK * q->K_o) / (q->K_o + q->K_mk)) * S[Na_i]) / (S[Na_i] + q->K_mNa) /
                       (1.00000 + 0.124500 * exp((-0.100000 * v * q->F) / RT) + 0.0353000 * exp((-v * q->F) / RT));
  const double E_Ca = ((0.500000 * q->R * q->T) / q->F) * log(q->Ca_o / S[Ca_i]);
  const double i_b_Ca = q->g_bca * (v - E_Ca);
  const double E_Na = ((q->R * q->T) / q->F) * log(q->Na_o / S[Na_i]);
  const double i_b_Na = q->g_bna * (v - E_Na);
  const double i_CaL = (((q->g_CaL * S[d] * S[f] * S[fCa] * 4.00000 * v * pow(q->F, 2.00000)) / RT) *
                        (S[Ca_i] * exp((2.00000 * v * q->F) / RT) - 0.341000 * q->Ca_o)) /
                       (exp((2.00000 * v * q->F) / RT) - 1.00000);
  const double alpha_d = 1.40000 / (1.00000 + exp((-35.0000 - v) / 13.0000)) + 0.250000;
  const double beta_d = 1.40000 / (1.00000 + exp((v + 5.00000) / 5.00000));
  const double gmma_d = 1.00000 / (1.00000 + exp((50.0000 - v) / 20.0000));
  const double tau_d = 1.00000 * alpha_d * beta_d + gmma_d;
  const double tau_f = 1125.00 * exp(-pow(v + 27.0000, 2.00000) / 240.000) + 80.0000 + 165.000 / (1.00000 + exp((25.0000 - v) / 10.0000));
  const double alpha_fCa = 1.00000 / (1.00000 + pow(S[Ca_i] / 0.000325000, 8.00000));
  const double beta_fCa = 0.100000 / (1.00000 + exp((S[Ca_i] - 0.000500000) / 0.000100000));
  const double gama_fCa = 0.200000 / (1.00000 + exp((S[Ca_i] - 0.000750000) / 0.000800000));
  const double d_inf = 1.00000 / (1.00000 + exp((-5.00000 - v) / 7.50000));
  const double f_inf = 1.00000 / (1.00000 + exp((v + 20.0000) / 7.00000));
  const double fCa_inf = (alpha_fCa + beta_fCa + gama_fCa + 0.230000) / 1.46000;
  const double d_fCa = (fCa_inf - S[fCa]) / q->tau_fCa;
  const double i_leak = q->V_leak * (S[Ca_SR] - S[Ca_i]);
  const double Ca_sr_bufsr = 1.00000 / (1.00000 + (q->Buf_sr * q->K_buf_sr) / pow(S[Ca_SR] + q->K_buf_sr, 2.00000));
  const double i_rel = ((q->a_rel * pow(S[Ca_SR], 2.00000)) / (pow(q->b_rel, 2.00000) + pow(S[Ca_SR], 2.00000)) + q->c_rel) * S[d] * S[g];
  const double g_inf = (S[Ca_i] < 0.000350000 ? 1.00000 / (1.00000 + pow(S[Ca_i] / 0.000350000, 6.00000))
                                              : 1.00000 / (1.00000 + pow(S[Ca_i] / 0.000350000, 16.0000)));
  const double d_g = (g_inf - S[g]) / q->tau_g;
  const double i_up = q->Vmax_up / (1.00000 + pow(q->K_up, 2.00000) / pow(S[Ca_i], 2.00000));
  const double E_K = ((q->R * q->T) / q->F) * log(q->K_o / S[K_i]);
  const double alpha_K1 = 0.100000 / (1.00000 + exp(0.0600000 * ((v - E_K) - 200.000)));
  const double beta_K1 = (3.00000 * exp(0.000200000 * ((v - E_K) + 100.000)) + 1.00000 * exp(0.100000 * ((v - E_K) - 10.0000))) /
                         (1.00000 + exp(-0.500000 * (v - E_K)));
  const double xK1_inf = alpha_K1 / (alpha_K1 + beta_K1);
  const double i_K1 = q->g_K1 * xK1_inf * pow((q->K_o / 5.40000), 1.0 / 2) * (v - E_K);
  const double i_Kr = q->g_Kr * pow((q->K_o / 5.40000), 1.0 / 2) * S[Xr1] * S[Xr2] * (v - E_K);
  const double alpha_xr1 = 450.000 / (1.00000 + exp((-45.0000 - v) / 10.0000));
  const double beta_xr1 = 6.00000 / (1.00000 + exp((v + 30.0000) / 11.5000));
  const double tau_xr1 = 1.00000 * alpha_xr1 * beta_xr1;
  const double alpha_xr2 = 3.00000 / (1.00000 + exp((-60.0000 - v) / 20.0000));
  const double beta_xr2 = 1.12000 / (1.00000 + exp((v - 60.0000) / 20.0000));
  const double tau_xr2 = 1.00000 * alpha_xr2 * beta_xr2;
  const double xr1_inf = 1.00000 / (1.00000 + exp((-26.0000 - v) / 7.00000));
  const double xr2_inf = 1.00000 / (1.00000 + exp((v + 88.0000) / 24.0000));
  const double E_Ks = ((q->R * q->T) / q->F) * log((q->K_o + q->P_kna * q->Na_o) / (S[K_i] + q->P_kna * S[Na_i]));
  const double i_Ks = q->g_Ks * pow(S[Xs], 2.00000) * (v - E_Ks);
  const double alpha_xs = 1100.00 / pow((1.00000 + exp((-10.0000 - v) / 6.00000)), 1.0 / 2);
  const double beta_xs = 1.00000 / (1.00000 + exp((v - 60.0000) / 20.0000));
  const double tau_xs = 1.00000 * alpha_xs * beta_xs;
  const double xs_inf = 1.00000 / (1.00000 + exp((-5.00000 - v) / 14.0000));
  const double i_Na = q->g_Na * pow(S[m], 3.00000) * S[h] * S[j] * (v - E_Na);
  const double m_inf = 1.00000 / pow(1.00000 + exp((-56.8600 - v) / 9.03000), 2.00000);
  const double h_inf = 1.00000 / pow(1.00000 + exp((v + 71.5500) / 7.43000), 2.00000);
  const double j_inf = 1.00000 / pow(1.00000 + exp((v + 71.5500) / 7.43000), 2.00000);
  const double alpha_m = 1.00000 / (1.00000 + exp((-60.0000 - v) / 5.00000));
  const double beta_m = 0.100000 / (1.00000 + exp((v + 35.0000) / 5.00000)) + 0.100000 / (1.00000 + exp((v - 50.0000) / 200.000));
  const double tau_m = 1.00000 * alpha_m * beta_m;
  const double alpha_h = (v < -40.0000 ? 0.0570000 * exp(-(v + 80.0000) / 6.80000) : 0.000000);
  const double beta_h = (v < -40.0000 ? 2.70000 * exp(0.0790000 * v) + 310000. * exp(0.348500 * v)
                                      : 0.770000 / (0.130000 * (1.00000 + exp((v + 10.6600) / -11.1000))));
  const double tau_h = 1.00000 / (alpha_h + beta_h);
  const double alpha_j = (v < -40.0000 ? (((-25428.0 * exp(0.244400 * v) - 6.94800e-06 * exp(-0.0439100 * v)) * (v + 37.7800)) / 1.00000) /
                                             (1.00000 + exp(0.311000 * (v + 79.2300)))
                                       : 0.000000);
  const double beta_j = (v < -40.0000 ? (0.0242400 * exp(-0.0105200 * v)) / (1.00000 + exp(-0.137800 * (v + 40.1400)))
                                      : (0.600000 * exp(0.0570000 * v)) / (1.00000 + exp(-0.100000 * (v + 32.0000))));
  const double tau_j = 1.00000 / (alpha_j + beta_j);
  const double i_p_K = (q->g_pK * (v - E_K)) / (1.00000 + exp((25.0000 - v) / 5.98000));
  const double i_p_Ca = (q->g_pCa * S[Ca_i]) / (S[Ca_i] + q->K_pCa);
  const double i_to = q->g_to * S[r] * S[s] * (v - E_K);
  const double tau_r = 9.50000 * exp(-pow(v + 40.0000, 2.00000) / 1800.00) + 0.800000;
  const double tau_s = 85.0000 * exp(-pow(v + 45.0000, 2.00000) / 320.000) + 5.00000 / (1.00000 + exp((v - 20.0000) / 5.00000)) + 3.00000;
  const double r_inf = 1.00000 / (1.00000 + exp((20.0000 - v) / 6.00000));
  const double s_inf = 1.00000 / (1.00000 + exp((v + 20.0000) / 5.00000));
  const double dV = -(i_K1 + i_to + i_Kr + i_Ks + i_CaL + i_NaK + i_Na + i_b_Na + i_NaCa + i_b_Ca + i_p_K + i_p_Ca + i_Stim);
  if (R_) {
    R_[V] = dV;
    R_[Na_i] = (-1.00000 * (i_Na + i_b_Na + 3.00000 * i_NaK + 3.00000 * i_NaCa) * q->Cm) / (1.00000 * q->V_c * q->F);
    R_[Ca_i] = Ca_i_bufc * (((i_leak - i_up) + i_rel) -
                            ((1.00000 * ((i_CaL + i_b_Ca + i_p_Ca) - 2.00000 * i_NaCa)) / (2.00000 * 1.00000 * q->V_c * q->F)) * q->Cm);
    R_[d] = (d_inf - S[d]) / tau_d;
    R_[f] = (f_inf - S[f]) / tau_f;
    R_[fCa] = (fCa_inf > S[fCa] && v > -60.0000 ? 0.000000 : d_fCa);
    R_[Ca_SR] = ((Ca_sr_bufsr * q->V_c) / q->V_sr) * (i_up - (i_rel + i_leak));
    R_[g] = (g_inf > S[g] && v > -60.0000 ? 0.000000 : d_g);
    R_[K_i] = (-1.00000 * ((i_K1 + i_to + i_Kr + i_Ks + i_p_K + i_Stim) - 2.00000 * i_NaK) * q->Cm) / (1.00000 * q->V_c * q->F);
    R_[Xr1] = (xr1_inf - S[Xr1]) / tau_xr1;
    R_[Xr2] = (xr2_inf - S[Xr2]) / tau_xr2;
    R_[Xs] = (xs_inf - S[Xs]) / tau_xs;
    R_[m] = (m_inf - S[m]) / tau_m;
    R_[h] = (h_inf - S[h]) / tau_h;
    R_[j] = (j_inf - S[j]) / tau_j;
    R_[r] = (r_inf - S[r]) / tau_r;
    R_[s] = (s_inf - S[s]) / tau_s;
  }
  if (al) {
    /* solveAnalytical's order: f, s, r, Xr1, Xr2, Xs, m, h, j, d */
    const double inf[10] = {f_inf, s_inf, r_inf, xr1_inf, xr2_inf, xs_inf, m_inf, h_inf, j_inf, d_inf};
    const double tau[10] = {tau_f, tau_s, tau_r, tau_xr1, tau_xr2, tau_xs, tau_m, tau_h, tau_j, tau_d};
    memcpy(al->inf, inf, sizeof(inf));
    memcpy(al->tau, tau, sizeof(tau));
  }
  if (cur) {
    cur->INa = i_Na; cur->INaL = 0.0; cur->Ito = i_to; cur->ICaL = i_CaL; cur->IKr = i_Kr; cur->IKs = i_Ks;
    cur->IK1 = i_K1; cur->dVdt = dV;
  }
}

void cepo_tt04_rates(const cepo_cell *c, double t, const double *y, double *dydt, cepo_currents *cur) {
  double r_[TT04_NS];
  tt04_compute(c, t, y, dydt ? dydt : r_, NULL, cur);
}

/* computeRates then solveAnalytical (:637-658) */
void cepo_tt04_step(const cepo_cell *c, double t, double dt, double *S, cepo_currents *cur) {
  double R_[TT04_NS];
  tt04_alg al;
  tt04_compute(c, t, S, R_, &al, cur);
  static const int idx[10] = {f, s, r, Xr1, Xr2, Xs, m, h, j, d};
  for (int k = 0; k < 10; ++k) S[idx[k]] = ((S[idx[k]] - al.inf[k]) * exp(-dt / al.tau[k])) + al.inf[k];
  S[g] += R_[g] * dt;
  S[fCa] += R_[fCa] * dt;
  S[Na_i] += R_[Na_i] * dt;
  S[V] += R_[V] * dt;
  S[K_i] += R_[K_i] * dt;
  S[Ca_i] += R_[Ca_i] * dt;
  S[Ca_SR] += R_[Ca_SR] * dt;
}

/* CONSTANTS[x] *= f after initConsts (population_tn2006.cpp:92-101,
 * anm_bench_custom.cpp:62-71): 0 g_Na, 2 g_to, 3 g_CaL, 4 g_Kr, 5 g_Ks,
 * 6 g_K1, 7 g_bna, 8 g_bca, 9 g_pCa, 10 g_pK. Returns -1 otherwise. */
int cepo_tt04_scale(cepo_cell *c, int g, double f) {
  tt04_p *q = (tt04_p *)c->p;
  double *x = g == 0 ? &q->g_Na : g == 2 ? &q->g_to : g == 3 ? &q->g_CaL : g == 4 ? &q->g_Kr : g == 5 ? &q->g_Ks
            : g == 6 ? &q->g_K1 : g == 7 ? &q->g_bna : g == 8 ? &q->g_bca : g == 9 ? &q->g_pCa : g == 10 ? &q->g_pK : 0;
  if (!x) return -1;
  *x *= f;
  return 0;
}
