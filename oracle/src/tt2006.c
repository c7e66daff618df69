/*
 * TEST INFRASTRUCTURE ONLY. CPU restatement of the ten Tusscher 2006
 * epicardial model (IK1 Ko-dependent variant) as CEPCell_NEO/cellmodels/
 * ten_tusscher_model_2006_IK1Ko_epi_units.cpp implements it: initConsts
 * (:196-272), computeRates (:274-380) and solveAnalytical (:382-407), in
 * the reference's evaluation order (pinned bit for bit against the reference
 * compiled from its own sources, single-cell and -DTISSUE builds).
 *
 * The reference model has no drug hook. The Hill block here follows the
 * reference's TT2004 hook (tentusscher_noble_noble_panfilov_2004_b.cpp:
 * 361-377): g_CaL, g_K1, g_Ks, g_Na, g_to, g_Kr scaled by
 * 1/(1 + (D/IC50)^h) from the CSV columns (0,1), (2,3), (4,5), (6,7),
 * (10,11), (12,13); INaL (8,9) has no counterpart in this model.
 */
#include <math.h>
#include <string.h>
#include "cep_oracle.h"

typedef struct {
  double R, T, F, Cm, V_c, stim_start, stim_period, stim_duration, stim_amplitude, P_kna, K_o, Na_o, Ca_o;
  double g_K1, g_Kr, g_Ks, g_Na, g_bna, g_CaL, g_bca, g_to, P_NaK, K_mk, K_mNa, K_NaCa, K_sat, alpha, gmma;
  double Km_Ca, Km_Nai, g_pCa, K_pCa, g_pK, k1_prime, k2_prime, k3, k4, EC, max_sr, min_sr, V_rel, V_xfer;
  double K_up, V_leak, Vmax_up, Buf_c, K_buf_c, Buf_sr, K_buf_sr, Buf_ss, K_buf_ss, V_sr, V_ss, tau_f_scale;
} tt06_p;

enum { V = 0, K_i, Na_i, Ca_i, Xr1, Xr2, Xs, m, h, j, Ca_ss, d, f, f2, fCass, s, r, Ca_SR, R_prime, TT06_NS };

static double hb(double D, double ic50, double hh) {
  return (ic50 > 10E-14 && hh > 10E-14) ? pow(1. + pow(D / ic50, hh), -1) : 1.;
}

int cepo_tt06_init(cepo_cell *c, double celltype, double conc, const double *hill, int is_dutta, int quirks) {
  (void)celltype; (void)is_dutta; (void)quirks;
  tt06_p *q = (tt06_p *)c->p;
  memset(c->p, 0, sizeof(c->p));
  q->R = 8314.472; q->T = 310; q->F = 96485.3415; q->Cm = 0.185; q->V_c = 0.016404; q->stim_start = 10;
  q->stim_period = 1000; q->stim_duration = 1; q->stim_amplitude = 52; q->P_kna = 0.03; q->K_o = 5.4;
  q->Na_o = 140; q->Ca_o = 2; q->g_K1 = 5.405; q->g_Kr = 0.153; q->g_Ks = 0.392; q->g_Na = 14.838;
  q->g_bna = 0.00029; q->g_CaL = 0.0000398; q->g_bca = 0.000592; q->g_to = 0.294; q->P_NaK = 2.724;
  q->K_mk = 1; q->K_mNa = 40; q->K_NaCa = 1000; q->K_sat = 0.1; q->alpha = 2.5; q->gmma = 0.35;
  q->Km_Ca = 1.38; q->Km_Nai = 87.5; q->g_pCa = 0.1238; q->K_pCa = 0.0005; q->g_pK = 0.0146;
  q->k1_prime = 0.15; q->k2_prime = 0.045; q->k3 = 0.06; q->k4 = 0.005; q->EC = 1.5; q->max_sr = 2.5;
  q->min_sr = 1; q->V_rel = 0.102; q->V_xfer = 0.0038; q->K_up = 0.00025; q->V_leak = 0.00036;
  q->Vmax_up = 0.006375; q->Buf_c = 0.2; q->K_buf_c = 0.001; q->Buf_sr = 10; q->K_buf_sr = 0.3;
  q->Buf_ss = 0.4; q->K_buf_ss = 0.00025; q->V_sr = 0.001094; q->V_ss = 0.00005468; q->tau_f_scale = 1.;
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

void cepo_tt06_init_states(double *y) {
  y[V] = -85.23; y[K_i] = 136.89; y[Na_i] = 8.604; y[Ca_i] = 0.000126; y[Xr1] = 0.00621; y[Xr2] = 0.4712;
  y[Xs] = 0.0095; y[m] = 0.00172; y[h] = 0.7444; y[j] = 0.7045; y[Ca_ss] = 0.00036; y[d] = 3.373e-5;
  y[f] = 0.7888; y[f2] = 0.9755; y[fCass] = 0.9953; y[s] = 0.999998; y[r] = 2.42e-8; y[Ca_SR] = 3.64;
  y[R_prime] = 0.9073;
}

void cepo_tt06_set_pacing(cepo_cell *c, double bcl, double stim_start, double stim_dur, double amp_scale) {
  tt06_p *q = (tt06_p *)c->p;
  q->stim_period = bcl;
  if (stim_start >= 0) q->stim_start = stim_start;
  if (stim_dur >= 0) q->stim_duration = stim_dur;
  q->stim_amplitude *= amp_scale;
}

void cepo_tt06_pacing(const cepo_cell *c, double *bcl, double *stim_start) {
  const tt06_p *q = (const tt06_p *)c->p;
  *bcl = q->stim_period;
  *stim_start = q->stim_start;
}

typedef struct {
  double inf[12], tau[12];  /* RL pairs in solveAnalytical's order */
  double iK1, ito, iKr, iKs, iCaL, iNaK, iNa, ibNa, iNaCa, ibCa, ipK, ipCa, iStim;
} tt06_alg;

/* computeRates, :274-380 */
static void tt06_compute(const cepo_cell *c, double TIME, const double *S, double *R_, tt06_alg *g,
                         cepo_currents *cur) {
  const tt06_p *q = (const tt06_p *)c->p;
  const double v = S[V];
  const double f_inf = 1.00000 / (1.00000 + exp((v + 20.0000) / 7.00000));
  const double tau_f = q->tau_f_scale * (1102.50 * exp(-pow(v + 27.0000, 2.00000) / 225.000) +
                                         200.000 / (1.00000 + exp((13.0000 - v) / 10.0000)) +
                                         180.000 / (1.00000 + exp((v + 30.0000) / 10.0000)) + 20.0000);
  const double f2_inf = 0.670000 / (1.00000 + exp((v + 35.0000) / 7.00000)) + 0.330000;
  const double tau_f2 = 562.000 * exp(-pow(v + 27.0000, 2.00000) / 240.000) + 31.0000 / (1.00000 + exp((25.0000 - v) / 10.0000)) +
                        80.0000 / (1.00000 + exp((v + 30.0000) / 10.0000));
  const double fCass_inf = 0.600000 / (1.00000 + pow(S[Ca_ss] / 0.0500000, 2.00000)) + 0.400000;
  const double tau_fCass = 80.0000 / (1.00000 + pow(S[Ca_ss] / 0.0500000, 2.00000)) + 2.00000;
  const double s_inf = 1.00000 / (1.00000 + exp((v + 20.0000) / 5.00000));
  const double tau_s = 85.0000 * exp(-pow(v + 45.0000, 2.00000) / 320.000) + 5.00000 / (1.00000 + exp((v - 20.0000) / 5.00000)) + 3.00000;
  const double r_inf = 1.00000 / (1.00000 + exp((20.0000 - v) / 6.00000));
  const double tau_r = 9.50000 * exp(-pow(v + 40.0000, 2.00000) / 1800.00) + 0.800000;
  const double xr1_inf = 1.00000 / (1.00000 + exp((-26.0000 - v) / 7.00000));
  const double alpha_xr1 = 450.000 / (1.00000 + exp((-45.0000 - v) / 10.0000));
  const double beta_xr1 = 6.00000 / (1.00000 + exp((v + 30.0000) / 11.5000));
  const double tau_xr1 = 1.00000 * alpha_xr1 * beta_xr1;
  const double xr2_inf = 1.00000 / (1.00000 + exp((v + 88.0000) / 24.0000));
  const double alpha_xr2 = 3.00000 / (1.00000 + exp((-60.0000 - v) / 20.0000));
  const double beta_xr2 = 1.12000 / (1.00000 + exp((v - 60.0000) / 20.0000));
  const double tau_xr2 = 1.00000 * alpha_xr2 * beta_xr2;
  const double xs_inf = 1.00000 / (1.00000 + exp((-5.00000 - v) / 14.0000));
  const double alpha_xs = 1400.00 / pow((1.00000 + exp((5.00000 - v) / 6.00000)), 1.0 / 2);
  const double beta_xs = 1.00000 / (1.00000 + exp((v - 35.0000) / 15.0000));
  const double tau_xs = 1.00000 * alpha_xs * beta_xs + 80.0000;
  const double m_inf = 1.00000 / pow(1.00000 + exp((-56.8600 - v) / 9.03000), 2.00000);
  const double alpha_m = 1.00000 / (1.00000 + exp((-60.0000 - v) / 5.00000));
  const double beta_m = 0.100000 / (1.00000 + exp((v + 35.0000) / 5.00000)) + 0.100000 / (1.00000 + exp((v - 50.0000) / 200.000));
  const double tau_m = 1.00000 * alpha_m * beta_m;
  const double h_inf = 1.00000 / pow(1.00000 + exp((v + 71.5500) / 7.43000), 2.00000);
  const double alpha_h = (v < -40.0000 ? 0.0570000 * exp(-(v + 80.0000) / 6.80000) : 0.000000);
  const double beta_h = (v < -40.0000 ? 2.70000 * exp(0.0790000 * v) + 310000. * exp(0.348500 * v)
                                      : 0.770000 / (0.130000 * (1.00000 + exp((v + 10.6600) / -11.1000))));
  const double tau_h = 1.00000 / (alpha_h + beta_h);
  const double j_inf = 1.00000 / pow(1.00000 + exp((v + 71.5500) / 7.43000), 2.00000);
  const double alpha_j = (v < -40.0000 ? (((-25428.0 * exp(0.244400 * v) - 6.94800e-06 * exp(-0.0439100 * v)) * (v + 37.7800)) / 1.00000) /
                                             (1.00000 + exp(0.311000 * (v + 79.2300)))
                                       : 0.000000);
  const double beta_j = (v < -40.0000 ? (0.0242400 * exp(-0.0105200 * v)) / (1.00000 + exp(-0.137800 * (v + 40.1400)))
                                      : (0.600000 * exp(0.0570000 * v)) / (1.00000 + exp(-0.100000 * (v + 32.0000))));
  const double tau_j = 1.00000 / (alpha_j + beta_j);
  const double d_inf = 1.00000 / (1.00000 + exp((-8.00000 - v) / 7.50000));
  const double alpha_d = 1.40000 / (1.00000 + exp((-35.0000 - v) / 13.0000)) + 0.250000;
  const double beta_d = 1.40000 / (1.00000 + exp((v + 5.00000) / 5.00000));
  const double gmma_d = 1.00000 / (1.00000 + exp((50.0000 - v) / 20.0000));
  const double tau_d = 1.00000 * alpha_d * beta_d + gmma_d;
  const double i_NaK = (((q->P_NaK * q->K_o) / (q->K_o + q->K_mk)) * S[Na_i]) / (S[Na_i] + q->K_mNa) /
                       (1.00000 + 0.124500 * exp((-0.100000 * v * q->F) / (q->R * q->T)) + 0.0353000 * exp((-v * q->F) / (q->R * q->T)));
  const double E_Na = ((q->R * q->T) / q->F) * log(q->Na_o / S[Na_i]);
  const double i_Na = q->g_Na * pow(S[m], 3.00000) * S[h] * S[j] * (v - E_Na);
  const double i_b_Na = q->g_bna * (v - E_Na);
  const double i_NaCa = (q->K_NaCa * (exp((q->gmma * v * q->F) / (q->R * q->T)) * pow(S[Na_i], 3.00000) * q->Ca_o -
                                      exp(((q->gmma - 1.00000) * v * q->F) / (q->R * q->T)) * pow(q->Na_o, 3.00000) * S[Ca_i] * q->alpha)) /
                        ((pow(q->Km_Nai, 3.00000) + pow(q->Na_o, 3.00000)) * (q->Km_Ca + q->Ca_o) *
                         (1.00000 + q->K_sat * exp(((q->gmma - 1.00000) * v * q->F) / (q->R * q->T))));
  const double E_K = ((q->R * q->T) / q->F) * log(q->K_o / S[K_i]);
  const double alpha_K1 = 0.100000 / (1.00000 + exp(0.0600000 * ((v - E_K) - 200.000)));
  const double beta_K1 = (3.00000 * exp(0.000200000 * ((v - E_K) + 100.000)) + exp(0.100000 * ((v - E_K) - 10.0000))) /
                         (1.00000 + exp(-0.500000 * (v - E_K)));
  const double xK1_inf = alpha_K1 / (alpha_K1 + beta_K1);
  const double i_K1 = q->g_K1 * xK1_inf * pow((q->K_o / 5.40000), 1.0 / 2) * (v - E_K);
  const double i_to = q->g_to * S[r] * S[s] * (v - E_K);
  const double i_Kr = q->g_Kr * pow((q->K_o / 5.40000), 1.0 / 2) * S[Xr1] * S[Xr2] * (v - E_K);
  const double E_Ks = ((q->R * q->T) / q->F) * log((q->K_o + q->P_kna * q->Na_o) / (S[K_i] + q->P_kna * S[Na_i]));
  const double i_Ks = q->g_Ks * pow(S[Xs], 2.00000) * (v - E_Ks);
  const double i_CaL = (((q->g_CaL * S[d] * S[f] * S[f2] * S[fCass] * 4.00000 * (v - 15.0000) * pow(q->F, 2.00000)) / (q->R * q->T)) *
                        (0.250000 * S[Ca_ss] * exp((2.00000 * (v - 15.0000) * q->F) / (q->R * q->T)) - q->Ca_o)) /
                       (exp((2.00000 * (v - 15.0000) * q->F) / (q->R * q->T)) - 1.00000);
  const double E_Ca = ((0.500000 * q->R * q->T) / q->F) * log(q->Ca_o / S[Ca_i]);
  const double i_b_Ca = q->g_bca * (v - E_Ca);
  const double i_p_K = (q->g_pK * (v - E_K)) / (1.00000 + exp((25.0000 - v) / 5.98000));
  const double i_p_Ca = (q->g_pCa * S[Ca_i]) / (S[Ca_i] + q->K_pCa);
  double i_Stim;
  if (c->tissue_stim) {
    i_Stim = c->is_s1 ? -q->stim_amplitude : 0.0;
  } else {
    i_Stim = (TIME - floor(TIME / q->stim_period) * q->stim_period >= q->stim_start &&
                      TIME - floor(TIME / q->stim_period) * q->stim_period <= q->stim_start + q->stim_duration
                  ? -q->stim_amplitude
                  : 0.000000);
  }
  const double i_up = q->Vmax_up / (1.00000 + pow(q->K_up, 2.00000) / pow(S[Ca_i], 2.00000));
  const double i_leak = q->V_leak * (S[Ca_SR] - S[Ca_i]);
  const double i_xfer = q->V_xfer * (S[Ca_ss] - S[Ca_i]);
  const double Ca_i_bufc = 1.00000 / (1.00000 + (q->Buf_c * q->K_buf_c) / pow(S[Ca_i] + q->K_buf_c, 2.00000));
  const double kcasr = q->max_sr - (q->max_sr - q->min_sr) / (1.00000 + pow(q->EC / S[Ca_SR], 2.00000));
  const double k2 = q->k2_prime * kcasr;
  const double k1 = q->k1_prime / kcasr;
  const double O = (k1 * pow(S[Ca_ss], 2.00000) * S[R_prime]) / (q->k3 + k1 * pow(S[Ca_ss], 2.00000));
  const double i_rel = q->V_rel * O * (S[Ca_SR] - S[Ca_ss]);
  const double Ca_sr_bufsr = 1.00000 / (1.00000 + (q->Buf_sr * q->K_buf_sr) / pow(S[Ca_SR] + q->K_buf_sr, 2.00000));
  const double Ca_ss_bufss = 1.00000 / (1.00000 + (q->Buf_ss * q->K_buf_ss) / pow(S[Ca_ss] + q->K_buf_ss, 2.00000));
  if (R_) {
    R_[f] = (f_inf - S[f]) / tau_f;
    R_[f2] = (f2_inf - S[f2]) / tau_f2;
    R_[fCass] = (fCass_inf - S[fCass]) / tau_fCass;
    R_[s] = (s_inf - S[s]) / tau_s;
    R_[r] = (r_inf - S[r]) / tau_r;
    R_[Xr1] = (xr1_inf - S[Xr1]) / tau_xr1;
    R_[Xr2] = (xr2_inf - S[Xr2]) / tau_xr2;
    R_[Xs] = (xs_inf - S[Xs]) / tau_xs;
    R_[m] = (m_inf - S[m]) / tau_m;
    R_[h] = (h_inf - S[h]) / tau_h;
    R_[j] = (j_inf - S[j]) / tau_j;
    R_[d] = (d_inf - S[d]) / tau_d;
    R_[Na_i] = ((-1.00000 * (i_Na + i_b_Na + 3.00000 * i_NaK + 3.00000 * i_NaCa)) / (1.00000 * q->V_c * q->F)) * q->Cm;
    R_[V] = (-1.00000 / 1.00000) * (i_K1 + i_to + i_Kr + i_Ks + i_CaL + i_NaK + i_Na + i_b_Na + i_NaCa + i_b_Ca + i_p_K + i_p_Ca + i_Stim);
    R_[K_i] = ((-1.00000 * ((i_K1 + i_to + i_Kr + i_Ks + i_p_K + i_Stim) - 2.00000 * i_NaK)) / (1.00000 * q->V_c * q->F)) * q->Cm;
    R_[Ca_i] = Ca_i_bufc * ((((i_leak - i_up) * q->V_sr) / q->V_c + i_xfer) -
                            (1.00000 * ((i_b_Ca + i_p_Ca) - 2.00000 * i_NaCa) * q->Cm) / (2.00000 * 1.00000 * q->V_c * q->F));
    R_[R_prime] = -k2 * S[Ca_ss] * S[R_prime] + q->k4 * (1.00000 - S[R_prime]);
    R_[Ca_SR] = Ca_sr_bufsr * (i_up - (i_rel + i_leak));
    R_[Ca_ss] = Ca_ss_bufss * (((-1.00000 * i_CaL * q->Cm) / (2.00000 * 1.00000 * q->V_ss * q->F) + (i_rel * q->V_sr) / q->V_ss) -
                               (i_xfer * q->V_c) / q->V_ss);
  }
  if (g) {
    const double inf[12] = {f_inf, f2_inf, fCass_inf, s_inf, r_inf, xr1_inf, xr2_inf, xs_inf, m_inf, h_inf, j_inf, d_inf};
    const double tau[12] = {tau_f, tau_f2, tau_fCass, tau_s, tau_r, tau_xr1, tau_xr2, tau_xs, tau_m, tau_h, tau_j, tau_d};
    memcpy(g->inf, inf, sizeof(inf));
    memcpy(g->tau, tau, sizeof(tau));
    g->iK1 = i_K1; g->ito = i_to; g->iKr = i_Kr; g->iKs = i_Ks; g->iCaL = i_CaL; g->iNaK = i_NaK; g->iNa = i_Na;
    g->ibNa = i_b_Na; g->iNaCa = i_NaCa; g->ibCa = i_b_Ca; g->ipK = i_p_K; g->ipCa = i_p_Ca; g->iStim = i_Stim;
  }
  if (cur) {
    cur->INa = i_Na; cur->INaL = 0.0; cur->Ito = i_to; cur->ICaL = i_CaL; cur->IKr = i_Kr; cur->IKs = i_Ks;
    cur->IK1 = i_K1; cur->dVdt = R_ ? R_[V] : 0.0;
  }
}

void cepo_tt06_rates(const cepo_cell *c, double t, const double *y, double *dydt, cepo_currents *cur) {
  double r_[TT06_NS];
  tt06_compute(c, t, y, dydt ? dydt : r_, NULL, cur);
}

/* computeRates then solveAnalytical (:382-407) */
void cepo_tt06_step(const cepo_cell *c, double t, double dt, double *S, cepo_currents *cur) {
  double R_[TT06_NS];
  tt06_alg g;
  tt06_compute(c, t, S, R_, &g, cur);
  static const int idx[12] = {f, f2, fCass, s, r, Xr1, Xr2, Xs, m, h, j, d};
  for (int k = 0; k < 12; ++k) S[idx[k]] = ((S[idx[k]] - g.inf[k]) * exp(-dt / g.tau[k])) + g.inf[k];
  S[V] = S[V] + (dt * -(g.iK1 + g.ito + g.iKr + g.iKs + g.iCaL + g.iNaK + g.iNa + g.ibNa + g.iNaCa + g.ibCa + g.ipK +
                        g.ipCa + g.iStim));
  S[R_prime] = S[R_prime] + R_[R_prime] * dt;
  S[Na_i] = S[Na_i] + R_[Na_i] * dt;
  S[K_i] = S[K_i] + R_[K_i] * dt;
  S[Ca_SR] = S[Ca_SR] + R_[Ca_SR] * dt;
  S[Ca_ss] = S[Ca_ss] + R_[Ca_ss] * dt;
  S[Ca_i] = S[Ca_i] + R_[Ca_i] * dt;
}

/* CONSTANTS[x] *= f after initConsts (population_tn2006.cpp:92-101,
 * anm_bench_custom.cpp:62-71): 0 g_Na, 2 g_to, 3 g_CaL, 4 g_Kr, 5 g_Ks,
 * 6 g_K1, 7 g_bna, 8 g_bca, 9 g_pCa, 10 g_pK. Returns -1 otherwise. */
int cepo_tt06_scale(cepo_cell *c, int g, double f) {
  tt06_p *q = (tt06_p *)c->p;
  double *x = g == 0 ? &q->g_Na : g == 2 ? &q->g_to : g == 3 ? &q->g_CaL : g == 4 ? &q->g_Kr : g == 5 ? &q->g_Ks
            : g == 6 ? &q->g_K1 : g == 7 ? &q->g_bna : g == 8 ? &q->g_bca : g == 9 ? &q->g_pCa : g == 10 ? &q->g_pK : 0;
  if (!x) return -1;
  *x *= f;
  return 0;
}
