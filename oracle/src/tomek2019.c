/*
 * TEST INFRASTRUCTURE ONLY. CPU restatement of the ToR-ORd model (Tomek et
 * al. 2019) as CEPCell_NEO/cellmodels/Tomek_model.cpp implements it:
 * ___initEndo / ___initEpi / ___initMid (:506-1134), the Hill hook
 * initConsts(celltype, conc, hill) (:1149-1168) and computeRates
 * (:1171-1440), in the reference's evaluation order (RATES pinned bit for
 * bit against the reference compiled from its own sources).
 *
 * The reference's solveAnalytical is empty (:1441-1443): it integrates this
 * model only with CVODE. The fixed-step scheme here is the reference's ORd
 * scheme (DrugSimulation/cellmodels/Ohara_Rudy_2011.cpp:1036-1094) carried
 * over: Rush-Larsen for every gate of the form (inf - y)/tau (including the
 * Jrel relaxations and nca with inf = anca k2n/km2n, tau = 1/km2n), forward
 * Euler for CaMKt, the IKr Markov states, V and the concentrations.
 *
 * Quirk (as ORd): the Hill hook scales PCa after PCap, PCaNa, PCaK, PCaNap
 * and PCaKp were derived from it, so the block does not reach them. With
 * quirks off they are re-derived from the blocked PCa.
 */
#include <math.h>
#include <string.h>
#include "cep_oracle.h"

typedef struct {
  double celltype, nao, cao, ko, clo, R, T, F, zna, zca, zk, zcl, L, rad, stim_start, stim_end, amp, BCL, duration;
  double KmCaMK, aCaMK, bCaMK, CaMKo, KmCaM, cmdnmax_b, kmcmdn, trpnmax, kmtrpn, BSRmax, KmBSR, BSLmax, KmBSL;
  double csqnmax, kmcsqn, cli, PKNa, gkatp, fkatp, K_o_n, A_atp, K_atp, GNa, thL, GNaL_b, Gto_b, EKshift, Kmn;
  double k2n, PCa_b, Aff, tjca, vShift, offset, dielConstant, ICaL_fractionSS, GKr_b, alpha_1, beta_1, GKs_b;
  double GK1_b, INaCa_fractionSS, kna1, kna2, kna3, kasymm, wna, wca, wnaca, kcaon, kcaoff, qna, qca, KmCaAct;
  double Gncx_b, k1p, k1m, k2p, k2m, k3p, k3m, k4p, k4m, Knai0, Knao0, delta, Kki, Kko, MgADP, MgATP, Kmgatp, H;
  double eP, Khp, Knap, Kxkur, Pnak_b, GKb_b, PNab, PCab, GpCa, KmCap, GClCa, GClb, KdClCa, Fjunc, tauNa, tauK;
  double tauCa, bt, cajsr_half, Jrel_b, Jup_b;
  /* derived (:690-713) */
  double vcell, cmdnmax, ECl, akik, bkik, thLp, GNaL, Gto, Afs, PCa, Io, GKr, GKs, GK1, GKb, a_rel, btp, upScale;
  double Ageo, PCap, PCaNa, PCaK, constA, a_relp, Acap, PCaNap, PCaKp, gamma_cao, gamma_nao, gamma_ko, vmyo, vnsr;
  double vjsr, vss, h10_i, h11_i, h12_i, k1_i, k2_i, k5_i, Gncx, h10_ss, h11_ss, h12_ss, k1_ss, k2_ss, k5_ss, b1;
  double a2, a4, Pnak;
} tomek_p;

enum {
  V = 0, CaMKt, cass, nai, nass, ki, kss, cansr, cajsr, cai, m, h, j, hp, jp, mL, hL, hLp, a, iF, iS, ap, iFp, iSp,
  d, ff, fs, fcaf, fcas, jca, ffp, fcafp, nca_ss, nca_i, C1, C2, C3, I, O, xs1, xs2, Jrel_np, Jrel_p, TOMEK_NS
};

static double hb(double D, double ic50, double hh) {
  return (ic50 > 10E-14 && hh > 10E-14) ? pow(1. + pow(D / ic50, hh), -1) : 1.;
}

static void base_consts(tomek_p *q, double celltype) {
  q->celltype = celltype; q->nao = 140.0; q->cao = 1.8; q->ko = 5.0; q->clo = 150.0; q->R = 8314; q->T = 310;
  q->F = 96485; q->zna = 1; q->zca = 2; q->zk = 1; q->zcl = -1; q->L = 0.01; q->rad = 0.0011;
  q->stim_start = 10; q->stim_end = 100000000000000000; q->amp = -53; q->BCL = 1000; q->duration = 1.0;
  q->KmCaMK = 0.15; q->aCaMK = 0.05; q->bCaMK = 0.00068; q->CaMKo = 0.05; q->KmCaM = 0.0015;
  q->cmdnmax_b = 0.05; q->kmcmdn = 0.00238; q->trpnmax = 0.07; q->kmtrpn = 0.0005; q->BSRmax = 0.047;
  q->KmBSR = 0.00087; q->BSLmax = 1.124; q->KmBSL = 0.0087; q->csqnmax = 10; q->kmcsqn = 0.8; q->cli = 24.0;
  q->PKNa = 0.01833; q->gkatp = 4.3195; q->fkatp = 0.0; q->K_o_n = 5; q->A_atp = 2; q->K_atp = 0.25;
  q->GNa = 11.7802; q->thL = 200; q->GNaL_b = 0.0279; q->Gto_b = 0.16; q->EKshift = 0; q->Kmn = 0.002;
  q->k2n = 500; q->PCa_b = 8.3757e-05; q->Aff = 0.6; q->tjca = 75; q->vShift = 0; q->offset = 0;
  q->dielConstant = 74; q->ICaL_fractionSS = 0.8; q->GKr_b = 0.0321; q->alpha_1 = 0.154375; q->beta_1 = 0.1911;
  q->GKs_b = 0.0011; q->GK1_b = 0.6992; q->INaCa_fractionSS = 0.35; q->kna1 = 15; q->kna2 = 5; q->kna3 = 88.12;
  q->kasymm = 12.5; q->wna = 6e4; q->wca = 6e4; q->wnaca = 5e3; q->kcaon = 1.5e6; q->kcaoff = 5e3; q->qna = 0.5224;
  q->qca = 0.167; q->KmCaAct = 150e-6; q->Gncx_b = 0.0034; q->k1p = 949.5; q->k1m = 182.4; q->k2p = 687.2;
  q->k2m = 39.4; q->k3p = 1899; q->k3m = 79300; q->k4p = 639; q->k4m = 40; q->Knai0 = 9.073; q->Knao0 = 27.78;
  q->delta = -0.155; q->Kki = 0.5; q->Kko = 0.3582; q->MgADP = 0.05; q->MgATP = 9.8; q->Kmgatp = 1.698e-7;
  q->H = 1e-7; q->eP = 4.2; q->Khp = 1.698e-7; q->Knap = 224; q->Kxkur = 292; q->Pnak_b = 15.4509;
  q->GKb_b = 0.0189; q->PNab = 1.9239e-09; q->PCab = 5.9194e-08; q->GpCa = 5e-04; q->KmCap = 0.0005;
  q->GClCa = 0.2843; q->GClb = 1.98e-3; q->KdClCa = 0.1; q->Fjunc = 1; q->tauNa = 2.0; q->tauK = 2.0;
  q->tauCa = 0.2; q->bt = 4.75; q->cajsr_half = 1.7; q->Jrel_b = 1.5378; q->Jup_b = 1.0;
  const double ct = q->celltype;
  q->vcell = 1000.00 * 3.14000 * q->rad * q->rad * q->L;
  q->cmdnmax = (ct == 1.00000 ? q->cmdnmax_b * 1.30000 : q->cmdnmax_b);
  q->ECl = ((q->R * q->T) / (q->zcl * q->F)) * log(q->clo / q->cli);
  q->akik = pow(q->ko / q->K_o_n, 0.240000);
  q->bkik = 1.00000 / (1.00000 + pow(q->A_atp / q->K_atp, 2.00000));
  q->thLp = 3.00000 * q->thL;
  q->GNaL = (ct == 1.00000 ? q->GNaL_b * 0.600000 : q->GNaL_b);
  q->Gto = (ct == 1.00000 ? q->Gto_b * 2.00000 : ct == 2.00000 ? q->Gto_b * 2.00000 : q->Gto_b);
  q->Afs = 1.00000 - q->Aff;
  q->PCa = (ct == 1.00000 ? q->PCa_b * 1.20000 : ct == 2.00000 ? q->PCa_b * 2.00000 : q->PCa_b);
  q->Io = (0.500000 * (q->nao + q->ko + q->clo + 4.00000 * q->cao)) / 1000.00;
  q->GKr = (ct == 1.00000 ? q->GKr_b * 1.30000 : ct == 2.00000 ? q->GKr_b * 0.800000 : q->GKr_b);
  q->GKs = (ct == 1.00000 ? q->GKs_b * 1.40000 : q->GKs_b);
  q->GK1 = (ct == 1.00000 ? q->GK1_b * 1.20000 : ct == 2.00000 ? q->GK1_b * 1.30000 : q->GK1_b);
  q->GKb = (ct == 1.00000 ? q->GKb_b * 0.600000 : q->GKb_b);
  q->a_rel = (0.500000 * q->bt) / 1.00000;
  q->btp = 1.25000 * q->bt;
  q->upScale = (ct == 1.00000 ? 1.30000 : 1.00000);
  q->Ageo = 2.00000 * 3.14000 * q->rad * q->rad + 2.00000 * 3.14000 * q->rad * q->L;
  q->PCap = 1.10000 * q->PCa;
  q->PCaNa = 0.00125000 * q->PCa;
  q->PCaK = 0.000357400 * q->PCa;
  q->constA = 1.82000e+06 * pow(q->dielConstant * q->T, -1.50000);
  q->a_relp = (0.500000 * q->btp) / 1.00000;
  q->Acap = 2.00000 * q->Ageo;
  q->PCaNap = 0.00125000 * q->PCap;
  q->PCaKp = 0.000357400 * q->PCap;
  const double sIo = pow(q->Io, 1.0 / 2);
  q->gamma_cao = exp(-q->constA * 4.00000 * (sIo / (1.00000 + sIo) - 0.300000 * q->Io));
  q->gamma_nao = exp(-q->constA * 1.00000 * (sIo / (1.00000 + sIo) - 0.300000 * q->Io));
  q->gamma_ko = exp(-q->constA * 1.00000 * (sIo / (1.00000 + sIo) - 0.300000 * q->Io));
  q->vmyo = 0.680000 * q->vcell;
  q->vnsr = 0.0552000 * q->vcell;
  q->vjsr = 0.00480000 * q->vcell;
  q->vss = 0.0200000 * q->vcell;
  q->h10_i = q->kasymm + 1.00000 + (q->nao / q->kna1) * (1.00000 + q->nao / q->kna2);
  q->h11_i = (q->nao * q->nao) / (q->h10_i * q->kna1 * q->kna2);
  q->h12_i = 1.00000 / q->h10_i;
  q->k1_i = q->h12_i * q->cao * q->kcaon;
  q->k2_i = q->kcaoff;
  q->k5_i = q->kcaoff;
  q->Gncx = (ct == 1.00000 ? q->Gncx_b * 1.10000 : ct == 2.00000 ? q->Gncx_b * 1.40000 : q->Gncx_b);
  q->h10_ss = q->kasymm + 1.00000 + (q->nao / q->kna1) * (1.00000 + q->nao / q->kna2);
  q->h11_ss = (q->nao * q->nao) / (q->h10_ss * q->kna1 * q->kna2);
  q->h12_ss = 1.00000 / q->h10_ss;
  q->k1_ss = q->h12_ss * q->cao * q->kcaon;
  q->k2_ss = q->kcaoff;
  q->k5_ss = q->kcaoff;
  q->b1 = q->k1m * q->MgADP;
  q->a2 = q->k2p;
  q->a4 = ((q->k4p * q->MgATP) / q->Kmgatp) / (1.00000 + q->MgATP / q->Kmgatp);
  q->Pnak = (ct == 1.00000 ? q->Pnak_b * 0.900000 : ct == 2.00000 ? q->Pnak_b * 0.700000 : q->Pnak_b);
}

int cepo_tomek_init(cepo_cell *c, double celltype, double conc, const double *hill, int is_dutta, int quirks) {
  (void)is_dutta;
  tomek_p *q = (tomek_p *)c->p;
  memset(c->p, 0, sizeof(c->p));
  /* celltype 0 endo, 1 epi, 2 mid (:1142-1147); anything else leaves the
   * constants unset in the reference; here it is rejected */
  if (celltype != 0. && celltype != 1. && celltype != 2.) return -2;
  base_consts(q, celltype);
  if (hill) {
    q->PCa *= hb(conc, hill[0], hill[1]);
    q->GK1 *= hb(conc, hill[2], hill[3]);
    q->GKs *= hb(conc, hill[4], hill[5]);
    q->GNa *= hb(conc, hill[6], hill[7]);
    q->GNaL *= hb(conc, hill[8], hill[9]);
    q->Gto *= hb(conc, hill[10], hill[11]);
    q->GKr *= hb(conc, hill[12], hill[13]);
    if (!quirks) {
      q->PCap = 1.10000 * q->PCa;
      q->PCaNa = 0.00125000 * q->PCa;
      q->PCaK = 0.000357400 * q->PCa;
      q->PCaNap = 0.00125000 * q->PCap;
      q->PCaKp = 0.000357400 * q->PCap;
    }
  }
  return 0;
}

void cepo_tomek_init_states(const cepo_cell *c, double *y) {
  static const double endo[TOMEK_NS] = {
      -88.7638, 0.0111, 7.0305e-5, 12.1025, 12.1029, 142.3002, 142.3002, 1.5211, 1.5214, 8.1583e-05, 8.0572e-4,
      0.8286, 0.8284, 0.6707, 0.8281, 1.629e-4, 0.5255, 0.2872, 9.5098e-4, 0.9996, 0.5936, 4.8454e-4, 0.9996,
      0.6538, 8.1084e-9, 1.0, 0.939, 1.0, 0.9999, 1.0, 1.0, 1.0, 6.6462e-4, 0.0012, 7.0344e-4, 8.5109e-4,
      0.9981, 1.3289e-5, 3.7585e-4, 0.248, 1.7707e-4, 1.6129e-22, 1.2475e-20};
  static const double epi[TOMEK_NS] = {
      -89.1400, 0.0129, 5.7672e-05, 12.8363, 12.8366, 142.6951, 142.6951, 1.8119, 1.8102, 6.6309e-05,
      0.00074303, 0.8360, 0.8359, 0.6828, 0.8357, 0.00015166, 0.5401, 0.3034, 0.00092716, 0.9996, 0.9996,
      0.0004724, 0.9996, 0.9996, 0, 1.0, 0.9485, 1.0, 0.9999, 1.0, 1.0, 1.0, 0.00030853, 0.00053006,
      0.00067941, 0.00082869, 0.9982, 9.5416e-06, 0.00027561, 0.2309, 0.00016975, 2.8189e-24, 0};
  static const double mid[TOMEK_NS] = {
      -89.1704, 0.0192, 6.5781e-05, 15.0038, 15.0043, 143.0403, 143.0402, 1.9557, 1.9593, 8.166e-05,
      0.00073818, 0.8365, 0.8363, 0.6838, 0.8358, 0.00015079, 0.5327, 0.2834, 0.00092527, 0.9996, 0.5671,
      0.00047143, 0.9996, 0.6261, 0, 1.0, 0.92, 1.0, 0.9998, 1.0, 1.0, 1.0, 0.00051399, 0.0012, 0.00069560,
      0.00082672, 0.9979, 1.8784e-05, 0.00054206, 0.2653, 0.00016921, 0, 0};
  const tomek_p *q = (const tomek_p *)c->p;
  memcpy(y, q->celltype == 1. ? epi : q->celltype == 2. ? mid : endo, sizeof(endo));
}

void cepo_tomek_set_pacing(cepo_cell *c, double bcl, double stim_start, double stim_dur, double amp_scale) {
  tomek_p *q = (tomek_p *)c->p;
  q->BCL = bcl;
  if (stim_start >= 0) q->stim_start = stim_start;
  if (stim_dur >= 0) q->duration = stim_dur;
  q->amp *= amp_scale;
}

void cepo_tomek_pacing(const cepo_cell *c, double *bcl, double *stim_start) {
  const tomek_p *q = (const tomek_p *)c->p;
  *bcl = q->BCL;
  *stim_start = q->stim_start;
}

/* one gate of the Rush-Larsen set: state index, steady state, time constant */
typedef struct {
  int n;
  int idx[32];
  double inf[32], tau[32];
} tomek_gates;

static void gate(tomek_gates *g, int idx, double inf, double tau) {
  g->idx[g->n] = idx;
  g->inf[g->n] = inf;
  g->tau[g->n] = tau;
  g->n++;
}

/* computeRates, :1171-1440 */
static void tomek_compute(const cepo_cell *c, double TIME, const double *S, double *R_, tomek_gates *gt,
                          cepo_currents *cur) {
  const tomek_p *q = (const tomek_p *)c->p;
  const double v = S[V];
  const double hLss = 1.00000 / (1.00000 + exp((v + 87.6100) / 7.48800));
  const double hLssp = 1.00000 / (1.00000 + exp((v + 93.8100) / 7.48800));
  const double jcass = 1.00000 / (1.00000 + exp((v + 18.0800) / 2.79160));
  const double mss = 1.00000 / pow(1.00000 + exp(-(v + 56.8600) / 9.03000), 2.00000);
  const double tm = 0.129200 * exp(-pow((v + 45.7900) / 15.5400, 2.00000)) + 0.0648700 * exp(-pow((v - 4.82300) / 51.1200, 2.00000));
  const double mLss = 1.00000 / (1.00000 + exp(-(v + 42.8500) / 5.26400));
  const double tmL = 0.129200 * exp(-pow((v + 45.7900) / 15.5400, 2.00000)) + 0.0648700 * exp(-pow((v - 4.82300) / 51.1200, 2.00000));
  const double ass = 1.00000 / (1.00000 + exp(-((v + q->EKshift) - 14.3400) / 14.8200));
  const double ta = 1.05150 / (1.00000 / (1.20890 * (1.00000 + exp(-((v + q->EKshift) - 18.4099) / 29.3814))) +
                               3.50000 / (1.00000 + exp((v + q->EKshift + 100.000) / 29.3814)));
  const double dss = (v >= 31.4978 ? 1.00000 : 1.07630 * exp(-1.00700 * exp(-0.0829000 * v)));
  const double td = q->offset + 0.600000 + 1.00000 / (exp(-0.0500000 * (v + q->vShift + 6.00000)) + exp(0.0900000 * (v + q->vShift + 14.0000)));
  const double fss = 1.00000 / (1.00000 + exp((v + 19.5800) / 3.69600));
  const double tff = 7.00000 + 1.00000 / (0.00450000 * exp(-(v + 20.0000) / 10.0000) + 0.00450000 * exp((v + 20.0000) / 10.0000));
  const double tfs = 1000.00 + 1.00000 / (3.50000e-05 * exp(-(v + 5.00000) / 4.00000) + 3.50000e-05 * exp((v + 5.00000) / 6.00000));
  const double km2n = S[jca] * 1.00000;
  const double anca_ss = 1.00000 / (q->k2n / km2n + pow(1.00000 + q->Kmn / S[cass], 4.00000));
  const double anca_i = 1.00000 / (q->k2n / km2n + pow(1.00000 + q->Kmn / S[cai], 4.00000));
  const double xs1ss = 1.00000 / (1.00000 + exp(-(v + 11.6000) / 8.93200));
  const double txs1 = 817.300 + 1.00000 / (0.000232600 * exp((v + 48.2800) / 17.8000) + 0.00129200 * exp(-(v + 210.000) / 230.000));
  const double assp = 1.00000 / (1.00000 + exp(-((v + q->EKshift) - 24.3400) / 14.8200));
  const double fcass = fss;
  const double tfcaf = 7.00000 + 1.00000 / (0.0400000 * exp(-(v - 4.00000) / 7.00000) + 0.0400000 * exp((v - 4.00000) / 7.00000));
  const double tfcas = 100.000 + 1.00000 / (0.000120000 * exp(-v / 3.00000) + 0.000120000 * exp(v / 7.00000));
  const double tffp = 2.50000 * tff;
  const double xs2ss = xs1ss;
  const double txs2 = 1.00000 / (0.0100000 * exp((v - 50.0000) / 20.0000) + 0.0193000 * exp(-(v + 66.5400) / 31.0000));
  const double CaMKb = (q->CaMKo * (1.00000 - S[CaMKt])) / (1.00000 + q->KmCaM / S[cass]);
  const double hss = 1.00000 / pow(1.00000 + exp((v + 71.5500) / 7.43000), 2.00000);
  const double ah = (v >= -40.0000 ? 0.00000 : 0.0570000 * exp(-(v + 80.0000) / 6.80000));
  const double bh = (v >= -40.0000 ? 0.770000 / (0.130000 * (1.00000 + exp(-(v + 10.6600) / 11.1000)))
                                   : 2.70000 * exp(0.0790000 * v) + 310000. * exp(0.348500 * v));
  const double th = 1.00000 / (ah + bh);
  const double tfcafp = 2.50000 * tfcaf;
  const double jss = hss;
  const double aj = (v >= -40.0000 ? 0.00000
                                   : ((-25428.0 * exp(0.244400 * v) - 6.94800e-06 * exp(-0.0439100 * v)) * (v + 37.7800)) /
                                         (1.00000 + exp(0.311000 * (v + 79.2300))));
  const double bj = (v >= -40.0000 ? (0.600000 * exp(0.0570000 * v)) / (1.00000 + exp(-0.100000 * (v + 32.0000)))
                                   : (0.0242400 * exp(-0.0105200 * v)) / (1.00000 + exp(-0.137800 * (v + 40.1400))));
  const double tj = 1.00000 / (aj + bj);
  const double hssp = 1.00000 / pow(1.00000 + exp((v + 77.5500) / 7.43000), 2.00000);
  const double iss = 1.00000 / (1.00000 + exp((v + q->EKshift + 43.9400) / 5.71100));
  const double delta_epi = (q->celltype == 1.00000 ? 1.00000 - 0.950000 / (1.00000 + exp((v + q->EKshift + 70.0000) / 5.00000)) : 1.00000);
  const double tiF_b = 4.56200 + 1.00000 / (0.393300 * exp(-(v + q->EKshift + 100.000) / 100.000) + 0.0800400 * exp((v + q->EKshift + 50.0000) / 16.5900));
  const double tiF = tiF_b * delta_epi;
  const double vfrt = (v * q->F) / (q->R * q->T);
  const double alpha = 0.116100 * exp(0.299000 * vfrt);
  const double beta = 0.244200 * exp(-1.60400 * vfrt);
  const double tjp = 1.46000 * tj;
  const double tiS_b = 23.6200 + 1.00000 / (0.00141600 * exp(-(v + q->EKshift + 96.5200) / 59.0500) + 1.78000e-08 * exp((v + q->EKshift + 114.100) / 8.07900));
  const double tiS = tiS_b * delta_epi;
  const double alpha_2 = 0.0578000 * exp(0.971000 * vfrt);
  const double beta_2 = 0.000349000 * exp(-1.06200 * vfrt);
  const double alpha_i = 0.253300 * exp(0.595300 * vfrt);
  const double beta_i = 0.0652500 * exp(-0.820900 * vfrt);
  const double dti_develop = 1.35400 + 0.000100000 / (exp(((v + q->EKshift) - 167.400) / 15.8900) + exp(-((v + q->EKshift) - 12.2300) / 0.215400));
  const double dti_recover = 1.00000 - 0.500000 / (1.00000 + exp((v + q->EKshift + 70.0000) / 20.0000));
  const double tiFp = dti_develop * dti_recover * tiF;
  const double tiSp = dti_develop * dti_recover * tiS;
  const double alpha_C2ToI = 5.20000e-05 * exp(1.52500 * vfrt);
  const double beta_ItoC2 = (beta_2 * beta_i * alpha_C2ToI) / (alpha_2 * alpha_i);
  const double f = q->Aff * S[ff] + q->Afs * S[fs];
  const double Afcaf = 0.300000 + 0.600000 / (1.00000 + exp((v - 10.0000) / 10.0000));
  const double Afcas = 1.00000 - Afcaf;
  const double fca = Afcaf * S[fcaf] + Afcas * S[fcas];
  const double fp = q->Aff * S[ffp] + q->Afs * S[fs];
  const double fcap = Afcaf * S[fcafp] + Afcas * S[fcas];
  const double vffrt = (v * q->F * q->F) / (q->R * q->T);
  const double Iss = (0.500000 * (S[nass] + S[kss] + q->cli + 4.00000 * S[cass])) / 1000.00;
  const double sIss = pow(Iss, 1.0 / 2);
  const double gamma_cass = exp(-q->constA * 4.00000 * (sIss / (1.00000 + sIss) - 0.300000 * Iss));
  const double PhiCaL_ss = (4.00000 * vffrt * (gamma_cass * S[cass] * exp(2.00000 * vfrt) - q->gamma_cao * q->cao)) / (exp(2.00000 * vfrt) - 1.00000);
  const double CaMKa = CaMKb + S[CaMKt];
  const double fICaLp = 1.00000 / (1.00000 + q->KmCaMK / CaMKa);
  const double ICaL_ss = q->ICaL_fractionSS * ((1.00000 - fICaLp) * q->PCa * PhiCaL_ss * S[d] * (f * (1.00000 - S[nca_ss]) + S[jca] * fca * S[nca_ss]) +
                                               fICaLp * q->PCap * PhiCaL_ss * S[d] * (fp * (1.00000 - S[nca_ss]) + S[jca] * fcap * S[nca_ss]));
  const double Jrel_inf_b = ((-q->a_rel * ICaL_ss) / 1.00000) / (1.00000 + pow(q->cajsr_half / S[cajsr], 8.00000));
  const double Jrel_inf = (q->celltype == 2.00000 ? Jrel_inf_b * 1.70000 : Jrel_inf_b);
  const double tau_rel_b = q->bt / (1.00000 + 0.0123000 / S[cajsr]);
  const double tau_rel = (tau_rel_b < 0.00100000 ? 0.00100000 : tau_rel_b);
  const double Jrel_infp_b = ((-q->a_relp * ICaL_ss) / 1.00000) / (1.00000 + pow(q->cajsr_half / S[cajsr], 8.00000));
  const double Jrel_infp = (q->celltype == 2.00000 ? Jrel_infp_b * 1.70000 : Jrel_infp_b);
  const double tau_relp_b = q->btp / (1.00000 + 0.0123000 / S[cajsr]);
  const double tau_relp = (tau_relp_b < 0.00100000 ? 0.00100000 : tau_relp_b);
  const double EK = ((q->R * q->T) / (q->zk * q->F)) * log(q->ko / S[ki]);
  const double AiF = 1.00000 / (1.00000 + exp(((v + q->EKshift) - 213.600) / 151.200));
  const double AiS = 1.00000 - AiF;
  const double i_ = AiF * S[iF] + AiS * S[iS];
  const double ip = AiF * S[iFp] + AiS * S[iSp];
  const double fItop = 1.00000 / (1.00000 + q->KmCaMK / CaMKa);
  const double Ito = q->Gto * (v - EK) * ((1.00000 - fItop) * S[a] * i_ + fItop * S[ap] * ip);
  const double IKr = q->GKr * pow((q->ko / 5.00000), 1.0 / 2) * S[O] * (v - EK);
  const double EKs = ((q->R * q->T) / (q->zk * q->F)) * log((q->ko + q->PKNa * q->nao) / (S[ki] + q->PKNa * S[nai]));
  const double KsCa = 1.00000 + 0.600000 / (1.00000 + pow(3.80000e-05 / S[cai], 1.40000));
  const double IKs = q->GKs * KsCa * S[xs1] * S[xs2] * (v - EKs);
  const double aK1 = 4.09400 / (1.00000 + exp(0.121700 * ((v - EK) - 49.9340)));
  const double bK1 = (15.7200 * exp(0.0674000 * ((v - EK) - 3.25700)) + exp(0.0618000 * ((v - EK) - 594.310))) / (1.00000 + exp(-0.162900 * ((v - EK) + 14.2070)));
  const double K1ss = aK1 / (aK1 + bK1);
  const double IK1 = q->GK1 * pow((q->ko / 5.00000), 1.0 / 2) * K1ss * (v - EK);
  const double Knao = q->Knao0 * exp(((1.00000 - q->delta) * vfrt) / 3.00000);
  const double a3 = (q->k3p * pow(q->ko / q->Kko, 2.00000)) / ((pow(1.00000 + q->nao / Knao, 3.00000) + pow(1.00000 + q->ko / q->Kko, 2.00000)) - 1.00000);
  const double P_ = q->eP / (1.00000 + q->H / q->Khp + S[nai] / q->Knap + S[ki] / q->Kxkur);
  const double b3 = (q->k3m * P_ * q->H) / (1.00000 + q->MgATP / q->Kmgatp);
  const double Knai = q->Knai0 * exp((q->delta * vfrt) / 3.00000);
  const double a1 = (q->k1p * pow(S[nai] / Knai, 3.00000)) / ((pow(1.00000 + S[nai] / Knai, 3.00000) + pow(1.00000 + S[ki] / q->Kki, 2.00000)) - 1.00000);
  const double b2 = (q->k2m * pow(q->nao / Knao, 3.00000)) / ((pow(1.00000 + q->nao / Knao, 3.00000) + pow(1.00000 + q->ko / q->Kko, 2.00000)) - 1.00000);
  const double b4 = (q->k4m * pow(S[ki] / q->Kki, 2.00000)) / ((pow(1.00000 + S[nai] / Knai, 3.00000) + pow(1.00000 + S[ki] / q->Kki, 2.00000)) - 1.00000);
  const double x1 = q->a4 * a1 * q->a2 + b2 * b4 * b3 + q->a2 * b4 * b3 + b3 * a1 * q->a2;
  const double x2 = b2 * q->b1 * b4 + a1 * q->a2 * a3 + a3 * q->b1 * b4 + q->a2 * a3 * b4;
  const double x3 = q->a2 * a3 * q->a4 + b3 * b2 * q->b1 + b2 * q->b1 * q->a4 + a3 * q->a4 * q->b1;
  const double x4 = b4 * b3 * b2 + a3 * q->a4 * a1 + b2 * q->a4 * a1 + b3 * b2 * a1;
  const double E1 = x1 / (x1 + x2 + x3 + x4);
  const double E2 = x2 / (x1 + x2 + x3 + x4);
  const double JnakNa = 3.00000 * (E1 * a3 - E2 * b3);
  const double E3 = x3 / (x1 + x2 + x3 + x4);
  const double E4 = x4 / (x1 + x2 + x3 + x4);
  const double JnakK = 2.00000 * (E4 * q->b1 - E3 * a1);
  const double INaK = q->Pnak * (q->zna * JnakNa + q->zk * JnakK);
  const double xkb = 1.00000 / (1.00000 + exp(-(v - 10.8968) / 23.9871));
  const double IKb = q->GKb * xkb * (v - EK);
  const double I_katp = q->fkatp * q->gkatp * q->akik * q->bkik * (v - EK);
  double Istim;
  if (c->tissue_stim)
    Istim = c->is_s1 ? q->amp : 0.0;
  else
    Istim = (TIME >= q->stim_start && TIME <= q->stim_end &&
                     (TIME - q->stim_start) - floor((TIME - q->stim_start) / q->BCL) * q->BCL <= q->duration
                 ? q->amp
                 : 0.00000);
  const double Ii = (0.500000 * (S[nai] + S[ki] + q->cli + 4.00000 * S[cai])) / 1000.00;
  const double sIi = pow(Ii, 1.0 / 2);
  const double gamma_ki = exp(-q->constA * 1.00000 * (sIi / (1.00000 + sIi) - 0.300000 * Ii));
  const double PhiCaK_i = (1.00000 * vffrt * (gamma_ki * S[ki] * exp(1.00000 * vfrt) - q->gamma_ko * q->ko)) / (exp(1.00000 * vfrt) - 1.00000);
  const double ICaK_i = (1.00000 - q->ICaL_fractionSS) * ((1.00000 - fICaLp) * q->PCaK * PhiCaK_i * S[d] * (f * (1.00000 - S[nca_i]) + S[jca] * fca * S[nca_i]) +
                                                         fICaLp * q->PCaKp * PhiCaK_i * S[d] * (fp * (1.00000 - S[nca_i]) + S[jca] * fcap * S[nca_i]));
  const double JdiffK = (S[kss] - S[ki]) / q->tauK;
  const double gamma_kss = exp(-q->constA * 1.00000 * (sIss / (1.00000 + sIss) - 0.300000 * Iss));
  const double PhiCaK_ss = (1.00000 * vffrt * (gamma_kss * S[kss] * exp(1.00000 * vfrt) - q->gamma_ko * q->ko)) / (exp(1.00000 * vfrt) - 1.00000);
  const double ICaK_ss = q->ICaL_fractionSS * ((1.00000 - fICaLp) * q->PCaK * PhiCaK_ss * S[d] * (f * (1.00000 - S[nca_ss]) + S[jca] * fca * S[nca_ss]) +
                                               fICaLp * q->PCaKp * PhiCaK_ss * S[d] * (fp * (1.00000 - S[nca_ss]) + S[jca] * fcap * S[nca_ss]));
  const double ENa = ((q->R * q->T) / (q->zna * q->F)) * log(q->nao / S[nai]);
  const double fINap = 1.00000 / (1.00000 + q->KmCaMK / CaMKa);
  const double INa = q->GNa * (v - ENa) * pow(S[m], 3.00000) * ((1.00000 - fINap) * S[h] * S[j] + fINap * S[hp] * S[jp]);
  const double fINaLp = 1.00000 / (1.00000 + q->KmCaMK / CaMKa);
  const double INaL = q->GNaL * (v - ENa) * S[mL] * ((1.00000 - fINaLp) * S[hL] + fINaLp * S[hLp]);
  const double allo_i = 1.00000 / (1.00000 + pow(q->KmCaAct / S[cai], 2.00000));
  const double hna = exp(q->qna * vfrt);
  const double h7_i = 1.00000 + (q->nao / q->kna3) * (1.00000 + 1.00000 / hna);
  const double h8_i = q->nao / (q->kna3 * hna * h7_i);
  const double k3pp_i = h8_i * q->wnaca;
  const double h1_i = 1.00000 + (S[nai] / q->kna3) * (1.00000 + hna);
  const double h2_i = (S[nai] * hna) / (q->kna3 * h1_i);
  const double k4pp_i = h2_i * q->wnaca;
  const double h4_i = 1.00000 + (S[nai] / q->kna1) * (1.00000 + S[nai] / q->kna2);
  const double h5_i = (S[nai] * S[nai]) / (h4_i * q->kna1 * q->kna2);
  const double k7_i = h5_i * h2_i * q->wna;
  const double k8_i = h8_i * q->h11_i * q->wna;
  const double h9_i = 1.00000 / h7_i;
  const double k3p_i = h9_i * q->wca;
  const double k3_i = k3p_i + k3pp_i;
  const double hca = exp(q->qca * vfrt);
  const double h3_i = 1.00000 / h1_i;
  const double k4p_i = (h3_i * q->wca) / hca;
  const double k4_i = k4p_i + k4pp_i;
  const double h6_i = 1.00000 / h4_i;
  const double k6_i = h6_i * S[cai] * q->kcaon;
  const double x1_i = q->k2_i * k4_i * (k7_i + k6_i) + q->k5_i * k7_i * (q->k2_i + k3_i);
  const double x2_i = q->k1_i * k7_i * (k4_i + q->k5_i) + k4_i * k6_i * (q->k1_i + k8_i);
  const double x3_i = q->k1_i * k3_i * (k7_i + k6_i) + k8_i * k6_i * (q->k2_i + k3_i);
  const double x4_i = q->k2_i * k8_i * (k4_i + q->k5_i) + k3_i * q->k5_i * (q->k1_i + k8_i);
  const double E1_i = x1_i / (x1_i + x2_i + x3_i + x4_i);
  const double E2_i = x2_i / (x1_i + x2_i + x3_i + x4_i);
  const double E3_i = x3_i / (x1_i + x2_i + x3_i + x4_i);
  const double E4_i = x4_i / (x1_i + x2_i + x3_i + x4_i);
  const double JncxNa_i = (3.00000 * (E4_i * k7_i - E1_i * k8_i) + E3_i * k4pp_i) - E2_i * k3pp_i;
  const double JncxCa_i = E2_i * q->k2_i - E1_i * q->k1_i;
  const double INaCa_i = (1.00000 - q->INaCa_fractionSS) * q->Gncx * allo_i * (q->zna * JncxNa_i + q->zca * JncxCa_i);
  const double INab = (q->PNab * vffrt * (S[nai] * exp(vfrt) - q->nao)) / (exp(vfrt) - 1.00000);
  const double gamma_nai = exp(-q->constA * 1.00000 * (sIi / (1.00000 + sIi) - 0.300000 * Ii));
  const double PhiCaNa_i = (1.00000 * vffrt * (gamma_nai * S[nai] * exp(1.00000 * vfrt) - q->gamma_nao * q->nao)) / (exp(1.00000 * vfrt) - 1.00000);
  const double ICaNa_i = (1.00000 - q->ICaL_fractionSS) * ((1.00000 - fICaLp) * q->PCaNa * PhiCaNa_i * S[d] * (f * (1.00000 - S[nca_i]) + S[jca] * fca * S[nca_i]) +
                                                           fICaLp * q->PCaNap * PhiCaNa_i * S[d] * (fp * (1.00000 - S[nca_i]) + S[jca] * fcap * S[nca_i]));
  const double JdiffNa = (S[nass] - S[nai]) / q->tauNa;
  const double allo_ss = 1.00000 / (1.00000 + pow(q->KmCaAct / S[cass], 2.00000));
  const double h7_ss = 1.00000 + (q->nao / q->kna3) * (1.00000 + 1.00000 / hna);
  const double h8_ss = q->nao / (q->kna3 * hna * h7_ss);
  const double k3pp_ss = h8_ss * q->wnaca;
  const double h1_ss = 1.00000 + (S[nass] / q->kna3) * (1.00000 + hna);
  const double h2_ss = (S[nass] * hna) / (q->kna3 * h1_ss);
  const double k4pp_ss = h2_ss * q->wnaca;
  const double h4_ss = 1.00000 + (S[nass] / q->kna1) * (1.00000 + S[nass] / q->kna2);
  const double h5_ss = (S[nass] * S[nass]) / (h4_ss * q->kna1 * q->kna2);
  const double k7_ss = h5_ss * h2_ss * q->wna;
  const double k8_ss = h8_ss * q->h11_ss * q->wna;
  const double h9_ss = 1.00000 / h7_ss;
  const double k3p_ss = h9_ss * q->wca;
  const double k3_ss = k3p_ss + k3pp_ss;
  const double h3_ss = 1.00000 / h1_ss;
  const double k4p_ss = (h3_ss * q->wca) / hca;
  const double k4_ss = k4p_ss + k4pp_ss;
  const double h6_ss = 1.00000 / h4_ss;
  const double k6_ss = h6_ss * S[cass] * q->kcaon;
  const double x1_ss = q->k2_ss * k4_ss * (k7_ss + k6_ss) + q->k5_ss * k7_ss * (q->k2_ss + k3_ss);
  const double x2_ss = q->k1_ss * k7_ss * (k4_ss + q->k5_ss) + k4_ss * k6_ss * (q->k1_ss + k8_ss);
  const double x3_ss = q->k1_ss * k3_ss * (k7_ss + k6_ss) + k8_ss * k6_ss * (q->k2_ss + k3_ss);
  const double x4_ss = q->k2_ss * k8_ss * (k4_ss + q->k5_ss) + k3_ss * q->k5_ss * (q->k1_ss + k8_ss);
  const double E1_ss = x1_ss / (x1_ss + x2_ss + x3_ss + x4_ss);
  const double E2_ss = x2_ss / (x1_ss + x2_ss + x3_ss + x4_ss);
  const double E3_ss = x3_ss / (x1_ss + x2_ss + x3_ss + x4_ss);
  const double E4_ss = x4_ss / (x1_ss + x2_ss + x3_ss + x4_ss);
  const double JncxNa_ss = (3.00000 * (E4_ss * k7_ss - E1_ss * k8_ss) + E3_ss * k4pp_ss) - E2_ss * k3pp_ss;
  const double JncxCa_ss = E2_ss * q->k2_ss - E1_ss * q->k1_ss;
  const double INaCa_ss = q->INaCa_fractionSS * q->Gncx * allo_ss * (q->zna * JncxNa_ss + q->zca * JncxCa_ss);
  const double gamma_nass = exp(-q->constA * 1.00000 * (sIss / (1.00000 + sIss) - 0.300000 * Iss));
  const double PhiCaNa_ss = (1.00000 * vffrt * (gamma_nass * S[nass] * exp(1.00000 * vfrt) - q->gamma_nao * q->nao)) / (exp(1.00000 * vfrt) - 1.00000);
  const double ICaNa_ss = q->ICaL_fractionSS * ((1.00000 - fICaLp) * q->PCaNa * PhiCaNa_ss * S[d] * (f * (1.00000 - S[nca_ss]) + S[jca] * fca * S[nca_ss]) +
                                                fICaLp * q->PCaNap * PhiCaNa_ss * S[d] * (fp * (1.00000 - S[nca_ss]) + S[jca] * fcap * S[nca_ss]));
  const double Jdiff = (S[cass] - S[cai]) / q->tauCa;
  const double fJrelp = 1.00000 / (1.00000 + q->KmCaMK / CaMKa);
  const double Jrel = q->Jrel_b * ((1.00000 - fJrelp) * S[Jrel_np] + fJrelp * S[Jrel_p]);
  const double Bcass = 1.00000 / (1.00000 + (q->BSRmax * q->KmBSR) / pow(q->KmBSR + S[cass], 2.00000) + (q->BSLmax * q->KmBSL) / pow(q->KmBSL + S[cass], 2.00000));
  const double gamma_cai = exp(-q->constA * 4.00000 * (sIi / (1.00000 + sIi) - 0.300000 * Ii));
  const double PhiCaL_i = (4.00000 * vffrt * (gamma_cai * S[cai] * exp(2.00000 * vfrt) - q->gamma_cao * q->cao)) / (exp(2.00000 * vfrt) - 1.00000);
  const double ICaL_i = (1.00000 - q->ICaL_fractionSS) * ((1.00000 - fICaLp) * q->PCa * PhiCaL_i * S[d] * (f * (1.00000 - S[nca_i]) + S[jca] * fca * S[nca_i]) +
                                                         fICaLp * q->PCap * PhiCaL_i * S[d] * (fp * (1.00000 - S[nca_i]) + S[jca] * fcap * S[nca_i]));
  const double ICaL = ICaL_ss + ICaL_i;
  const double ICaNa = ICaNa_ss + ICaNa_i;
  const double ICaK = ICaK_ss + ICaK_i;
  const double IpCa = (q->GpCa * S[cai]) / (q->KmCap + S[cai]);
  const double ICab = (q->PCab * 4.00000 * vffrt * (gamma_cai * S[cai] * exp(2.00000 * vfrt) - q->gamma_cao * q->cao)) / (exp(2.00000 * vfrt) - 1.00000);
  const double IClCa_junc = ((q->Fjunc * q->GClCa) / (1.00000 + q->KdClCa / S[cass])) * (v - q->ECl);
  const double IClCa_sl = (((1.00000 - q->Fjunc) * q->GClCa) / (1.00000 + q->KdClCa / S[cai])) * (v - q->ECl);
  const double IClCa = IClCa_junc + IClCa_sl;
  const double IClb = q->GClb * (v - q->ECl);
  const double Jupnp = (q->upScale * 0.00542500 * S[cai]) / (S[cai] + 0.000920000);
  const double Jupp = (q->upScale * 2.75000 * 0.00542500 * S[cai]) / ((S[cai] + 0.000920000) - 0.000170000);
  const double fJupp = 1.00000 / (1.00000 + q->KmCaMK / CaMKa);
  const double Jleak = (0.00488250 * S[cansr]) / 15.0000;
  const double Jup = q->Jup_b * (((1.00000 - fJupp) * Jupnp + fJupp * Jupp) - Jleak);
  const double Bcai = 1.00000 / (1.00000 + (q->cmdnmax * q->kmcmdn) / pow(q->kmcmdn + S[cai], 2.00000) + (q->trpnmax * q->kmtrpn) / pow(q->kmtrpn + S[cai], 2.00000));
  const double Jtr = (S[cansr] - S[cajsr]) / 60.0000;
  const double Bcajsr = 1.00000 / (1.00000 + (q->csqnmax * q->kmcsqn) / pow(q->kmcsqn + S[cajsr], 2.00000));
  const double dV = -(INa + INaL + Ito + ICaL + ICaNa + ICaK + IKr + IKs + IK1 + INaCa_i + INaCa_ss + INaK + INab + IKb + IpCa + ICab +
                      IClCa + IClb + I_katp + Istim);
  if (R_) {
    R_[hL] = (hLss - S[hL]) / q->thL;
    R_[hLp] = (hLssp - S[hLp]) / q->thLp;
    R_[jca] = (jcass - S[jca]) / q->tjca;
    R_[m] = (mss - S[m]) / tm;
    R_[mL] = (mLss - S[mL]) / tmL;
    R_[a] = (ass - S[a]) / ta;
    R_[d] = (dss - S[d]) / td;
    R_[ff] = (fss - S[ff]) / tff;
    R_[fs] = (fss - S[fs]) / tfs;
    R_[nca_ss] = anca_ss * q->k2n - S[nca_ss] * km2n;
    R_[nca_i] = anca_i * q->k2n - S[nca_i] * km2n;
    R_[xs1] = (xs1ss - S[xs1]) / txs1;
    R_[ap] = (assp - S[ap]) / ta;
    R_[fcaf] = (fcass - S[fcaf]) / tfcaf;
    R_[fcas] = (fcass - S[fcas]) / tfcas;
    R_[ffp] = (fss - S[ffp]) / tffp;
    R_[xs2] = (xs2ss - S[xs2]) / txs2;
    R_[CaMKt] = q->aCaMK * CaMKb * (CaMKb + S[CaMKt]) - q->bCaMK * S[CaMKt];
    R_[h] = (hss - S[h]) / th;
    R_[fcafp] = (fcass - S[fcafp]) / tfcafp;
    R_[j] = (jss - S[j]) / tj;
    R_[hp] = (hssp - S[hp]) / th;
    R_[iF] = (iss - S[iF]) / tiF;
    R_[C3] = beta * S[C2] - alpha * S[C3];
    R_[C2] = (alpha * S[C3] + q->beta_1 * S[C1]) - (beta + q->alpha_1) * S[C2];
    R_[jp] = (jss - S[jp]) / tjp;
    R_[iS] = (iss - S[iS]) / tiS;
    R_[O] = (alpha_2 * S[C1] + beta_i * S[I]) - (beta_2 + alpha_i) * S[O];
    R_[iFp] = (iss - S[iFp]) / tiFp;
    R_[iSp] = (iss - S[iSp]) / tiSp;
    R_[C1] = (q->alpha_1 * S[C2] + beta_2 * S[O] + beta_ItoC2 * S[I]) - (q->beta_1 + alpha_2 + alpha_C2ToI) * S[C1];
    R_[I] = (alpha_C2ToI * S[C1] + alpha_i * S[O]) - (beta_ItoC2 + beta_i) * S[I];
    R_[Jrel_np] = (Jrel_inf - S[Jrel_np]) / tau_rel;
    R_[Jrel_p] = (Jrel_infp - S[Jrel_p]) / tau_relp;
    R_[ki] = (-(((Ito + IKr + IKs + IK1 + IKb + I_katp + Istim) - 2.00000 * INaK) + ICaK_i) * q->Acap) / (q->F * q->vmyo) + (JdiffK * q->vss) / q->vmyo;
    R_[kss] = (-ICaK_ss * q->Acap) / (q->F * q->vss) - JdiffK;
    R_[nai] = (-(INa + INaL + 3.00000 * INaCa_i + ICaNa_i + 3.00000 * INaK + INab) * q->Acap) / (q->F * q->vmyo) + (JdiffNa * q->vss) / q->vmyo;
    R_[nass] = (-(ICaNa_ss + 3.00000 * INaCa_ss) * q->Acap) / (q->F * q->vss) - JdiffNa;
    R_[cass] = Bcass * (((-(ICaL_ss - 2.00000 * INaCa_ss) * q->Acap) / (2.00000 * q->F * q->vss) + (Jrel * q->vjsr) / q->vss) - Jdiff);
    R_[V] = dV;
    R_[cai] = Bcai * (((-((ICaL_i + IpCa + ICab) - 2.00000 * INaCa_i) * q->Acap) / (2.00000 * q->F * q->vmyo) - (Jup * q->vnsr) / q->vmyo) +
                      (Jdiff * q->vss) / q->vmyo);
    R_[cansr] = Jup - (Jtr * q->vjsr) / q->vnsr;
    R_[cajsr] = Bcajsr * (Jtr - Jrel);
  }
  if (gt) {
    gt->n = 0;
    gate(gt, hL, hLss, q->thL); gate(gt, hLp, hLssp, q->thLp); gate(gt, jca, jcass, q->tjca);
    gate(gt, m, mss, tm); gate(gt, mL, mLss, tmL); gate(gt, a, ass, ta); gate(gt, d, dss, td);
    gate(gt, ff, fss, tff); gate(gt, fs, fss, tfs); gate(gt, xs1, xs1ss, txs1); gate(gt, ap, assp, ta);
    gate(gt, fcaf, fcass, tfcaf); gate(gt, fcas, fcass, tfcas); gate(gt, ffp, fss, tffp); gate(gt, xs2, xs2ss, txs2);
    gate(gt, h, hss, th); gate(gt, fcafp, fcass, tfcafp); gate(gt, j, jss, tj); gate(gt, hp, hssp, th);
    gate(gt, iF, iss, tiF); gate(gt, jp, jss, tjp); gate(gt, iS, iss, tiS); gate(gt, iFp, iss, tiFp);
    gate(gt, iSp, iss, tiSp); gate(gt, Jrel_np, Jrel_inf, tau_rel); gate(gt, Jrel_p, Jrel_infp, tau_relp);
    /* nca: dn/dt = anca k2n - n km2n */
    gate(gt, nca_ss, anca_ss * q->k2n / km2n, 1.00000 / km2n);
    gate(gt, nca_i, anca_i * q->k2n / km2n, 1.00000 / km2n);
  }
  if (cur) {
    cur->INa = INa; cur->INaL = INaL; cur->Ito = Ito; cur->ICaL = ICaL; cur->IKr = IKr; cur->IKs = IKs;
    cur->IK1 = IK1; cur->dVdt = dV;
  }
}

void cepo_tomek_rates(const cepo_cell *c, double t, const double *y, double *dydt, cepo_currents *cur) {
  double r_[TOMEK_NS];
  tomek_compute(c, t, y, dydt ? dydt : r_, NULL, cur);
}

/* Fixed step: Rush-Larsen gates, forward Euler for the rest */
void cepo_tomek_step(const cepo_cell *c, double t, double dt, double *S, cepo_currents *cur) {
  double R_[TOMEK_NS];
  tomek_gates g;
  tomek_compute(c, t, S, R_, &g, cur);
  for (int k = 0; k < g.n; ++k) S[g.idx[k]] = g.inf[k] - (g.inf[k] - S[g.idx[k]]) * exp(-dt / g.tau[k]);
  static const int fe[] = {V, CaMKt, cass, nai, nass, ki, kss, cansr, cajsr, cai, C1, C2, C3, I, O};
  for (unsigned k = 0; k < sizeof(fe) / sizeof(fe[0]); ++k) S[fe[k]] += R_[fe[k]] * dt;
}

/* CONSTANTS[x] *= f after initConsts, x one of the CEP scale conductances
 * (0 GNa, 1 GNaL, 2 Gto, 3 PCa, 4 GKr, 5 GKs, 6 GK1, 11 GKb, 12 Gncx,
 * 13 Pnak), as the reference's call sites do (cipa_drug_bench.cpp:148).
 * Returns -1 for a conductance the model has no constant for here. */
int cepo_tomek_scale(cepo_cell *c, int g, double f) {
  tomek_p *q = (tomek_p *)c->p;
  double *x = g == 0 ? &q->GNa : g == 1 ? &q->GNaL : g == 2 ? &q->Gto : g == 3 ? &q->PCa : g == 4 ? &q->GKr
            : g == 5 ? &q->GKs : g == 6 ? &q->GK1 : g == 11 ? &q->GKb : g == 12 ? &q->Gncx : g == 13 ? &q->Pnak : 0;
  if (!x) return -1;
  *x *= f;
  return 0;
}
