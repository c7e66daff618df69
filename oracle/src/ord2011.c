/*
 * TEST INFRASTRUCTURE ONLY. CPU restatement of the O'Hara-Rudy 2011 model as
 * the reference implements it in DrugSimulation/cellmodels/Ohara_Rudy_2011.cpp,
 * kept in the reference's evaluation order so that it reproduces the
 * reference bit for bit (pinned by tests/test_oracle_pin.py against the
 * reference compiled from its own sources).
 *
 * quirks = 1 reproduces the reference exactly:
 *   (1) solveAnalytical updates fcafp with exp(-d/tfcafp), d being the STATES
 *       enum value 25, not dt (Ohara_Rudy_2011.cpp:1064 of the reference file,
 *       the line `STATES[fcafp] = ... exp(-d / ALGEBRAIC[tfcafp])`);
 *   (2) ___initConsts resets CONSTANTS[celltype] to 0 after the caller set it
 *       (Ohara_Rudy_2011.cpp:496 vs :724), so every cell is endocardial;
 *   (3) ___applyDutta indexes CONSTANTS with ALGEBRAIC enum values
 *       (Ohara_Rudy_2011.cpp:460-467): it scales Aff, GNaL, tjca, H and
 *       Gncx_b instead of GKs, GKr, GK1, PCa and GNaL;
 *   (4) the drug block scales PCa after PCap/PCaNa/PCaK/PCaNap/PCaKp were
 *       derived from it (Ohara_Rudy_2011.cpp:471 vs :650-660), so only the
 *       non-phosphorylated Ca channel is blocked.
 * quirks = 0 gives the intended model (celltype honoured, Dutta scaling on
 * the named conductances, derived permeabilities re-derived, dt in fcafp).
 */
#include <math.h>
#include <string.h>
#include "cep_oracle.h"

typedef struct {
  double celltype, nao, cao, ko, R, T, F, zna, zca, zk, L, rad, stim_start, BCL, amp, duration;
  double KmCaMK, aCaMK, bCaMK, CaMKo, KmCaM, cmdnmax_b, kmcmdn, trpnmax, kmtrpn, BSRmax, KmBSR;
  double BSLmax, KmBSL, csqnmax, kmcsqn, cm, PKNa, mssV1, mssV2, mtV1, mtV2, mtD1, mtD2, mtV3, mtV4;
  double hssV1, hssV2, Ahf, GNa, thL, GNaL_b, Gto_b, Kmn, k2n, PCa_b, GKr_b, GKs_b, GK1_b;
  double kna1, kna2, kna3, kasymm, wna, wca, wnaca, kcaon, kcaoff, qna, qca, KmCaAct, Gncx_b;
  double k1p, k1m, k2p, k2m, k3p, k3m, k4p, k4m, Knai0, Knao0, delta, Kki, Kko, MgADP, MgATP;
  double Kmgatp, H, eP, Khp, Knap, Kxkur, Pnak_b, GKb_b, PNab, PCab, GpCa, KmCap, bt;
  /* derived */
  double cmdnmax, Ahs, thLp, GNaL, Gto, Aff, PCa, tjca, GKr, GKs, GK1, vcell, GKb, a_rel, btp;
  double upScale, Afs, PCap, PCaNa, PCaK, Ageo, a_relp, PCaNap, PCaKp, Acap, vmyo, vnsr, vjsr, vss;
  double h10_i, h11_i, h12_i, k1_i, k2_i, k5_i, Gncx, h10_ss, h11_ss, h12_ss, k1_ss, k2_ss, k5_ss;
  double b1, a2, a4, Pnak;
  double fcafp_dt; /* step used in the fcafp gate: 25 under quirk (1), else dt (0 = use dt) */
  double cumm_BCL; /* start of the current pace under the cumulative stimulus (hrv_bench) */
} ord_p;

_Static_assert(sizeof(ord_p) <= CEPO_MAX_PARAMS * sizeof(double), "ord_p too large");

/* STATES order of enums/enum_Ohara_Rudy_2011.hpp (the public interface). */
enum {
  V = 0, CaMKt, cass, nai, nass, ki, kss, cansr, cajsr, cai, m, hf, hs, j, hsp, jp, mL, hL, hLp, a,
  iF, iS, ap, iFp, iSp, d, ff, fs, fcaf, fcas, jca, ffp, fcafp, nca, xrf, xrs, xs1, xs2, xk1,
  Jrelnp, Jrelp, ORD_NS
};

static void derive_pca(ord_p *q) {
  q->PCap = 1.10000 * q->PCa;
  q->PCaNa = 0.00125000 * q->PCa;
  q->PCaK = 0.000357400 * q->PCa;
  q->PCaNap = 0.00125000 * q->PCap;
  q->PCaKp = 0.000357400 * q->PCap;
}

/* ___initConsts, Ohara_Rudy_2011.cpp:494-678. */
static void ord_base_consts(ord_p *q, double celltype) {
  q->celltype = celltype;
  q->nao = 140; q->cao = 1.8; q->ko = 5.4; q->R = 8314; q->T = 310; q->F = 96485;
  q->zna = 1; q->zca = 2; q->zk = 1; q->L = 0.01; q->rad = 0.0011;
  q->stim_start = 10.0; q->BCL = 1000.0; q->amp = -80; q->duration = 0.5;
  q->KmCaMK = 0.15; q->aCaMK = 0.05; q->bCaMK = 0.00068; q->CaMKo = 0.05; q->KmCaM = 0.0015;
  q->cmdnmax_b = 0.05; q->kmcmdn = 0.00238; q->trpnmax = 0.07; q->kmtrpn = 0.0005;
  q->BSRmax = 0.047; q->KmBSR = 0.00087; q->BSLmax = 1.124; q->KmBSL = 0.0087;
  q->csqnmax = 10; q->kmcsqn = 0.8; q->cm = 1; q->PKNa = 0.01833;
  q->mssV1 = 39.57; q->mssV2 = 9.871; q->mtV1 = 11.64; q->mtV2 = 34.77; q->mtD1 = 6.765;
  q->mtD2 = 8.552; q->mtV3 = 77.42; q->mtV4 = 5.955; q->hssV1 = 82.9; q->hssV2 = 6.086;
  q->Ahf = 0.99; q->GNa = 75; q->thL = 200; q->GNaL_b = 0.0075; q->Gto_b = 0.02;
  q->Kmn = 0.002; q->k2n = 1000; q->PCa_b = 0.0001; q->GKr_b = 0.046; q->GKs_b = 0.0034;
  q->GK1_b = 0.1908; q->kna1 = 15; q->kna2 = 5; q->kna3 = 88.12; q->kasymm = 12.5;
  q->wna = 6e4; q->wca = 6e4; q->wnaca = 5e3; q->kcaon = 1.5e6; q->kcaoff = 5e3;
  q->qna = 0.5224; q->qca = 0.167; q->KmCaAct = 150e-6; q->Gncx_b = 0.0008;
  q->k1p = 949.5; q->k1m = 182.4; q->k2p = 687.2; q->k2m = 39.4; q->k3p = 1899; q->k3m = 79300;
  q->k4p = 639; q->k4m = 40; q->Knai0 = 9.073; q->Knao0 = 27.78; q->delta = -0.155;
  q->Kki = 0.5; q->Kko = 0.3582; q->MgADP = 0.05; q->MgATP = 9.8; q->Kmgatp = 1.698e-7;
  q->H = 1e-7; q->eP = 4.2; q->Khp = 1.698e-7; q->Knap = 224; q->Kxkur = 292; q->Pnak_b = 30;
  q->GKb_b = 0.003; q->PNab = 3.75e-10; q->PCab = 2.5e-8; q->GpCa = 0.0005; q->KmCap = 0.0005;
  q->bt = 4.75;
  const double ct = q->celltype;
  q->cmdnmax = (ct == 1.0 ? q->cmdnmax_b * 1.30000 : q->cmdnmax_b);
  q->Ahs = 1.00000 - q->Ahf;
  q->thLp = 3.00000 * q->thL;
  q->GNaL = (ct == 1.0 ? q->GNaL_b * 0.600000 : q->GNaL_b);
  q->Gto = (ct == 1.0 ? q->Gto_b * 4.00000 : ct == 2.0 ? q->Gto_b * 4.00000 : q->Gto_b);
  q->Aff = 0.600000;
  q->PCa = (ct == 1.0 ? q->PCa_b * 1.20000 : ct == 2.0 ? q->PCa_b * 2.50000 : q->PCa_b);
  q->tjca = 75.0000;
  q->GKr = (ct == 1.0 ? q->GKr_b * 1.30000 : ct == 2.0 ? q->GKr_b * 0.800000 : q->GKr_b);
  q->GKs = (ct == 1.0 ? q->GKs_b * 1.40000 : q->GKs_b);
  q->GK1 = (ct == 1.0 ? q->GK1_b * 1.20000 : ct == 2.0 ? q->GK1_b * 1.30000 : q->GK1_b);
  q->vcell = 1000.00 * 3.14000 * q->rad * q->rad * q->L;
  q->GKb = (ct == 1.0 ? q->GKb_b * 0.600000 : q->GKb_b);
  q->a_rel = 0.500000 * q->bt;
  q->btp = 1.25000 * q->bt;
  q->upScale = (ct == 1.0 ? 1.30000 : 1.00000);
  q->Afs = 1.00000 - q->Aff;
  derive_pca(q);
  q->Ageo = 2.00000 * 3.14000 * q->rad * q->rad + 2.00000 * 3.14000 * q->rad * q->L;
  q->a_relp = 0.500000 * q->btp;
  q->Acap = 2.00000 * q->Ageo;
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
  q->Gncx = (ct == 1.0 ? q->Gncx_b * 1.10000 : ct == 2.0 ? q->Gncx_b * 1.40000 : q->Gncx_b);
  q->h10_ss = q->kasymm + 1.00000 + (q->nao / q->kna1) * (1.00000 + q->nao / q->kna2);
  q->h11_ss = (q->nao * q->nao) / (q->h10_ss * q->kna1 * q->kna2);
  q->h12_ss = 1.00000 / q->h10_ss;
  q->k1_ss = q->h12_ss * q->cao * q->kcaon;
  q->k2_ss = q->kcaoff;
  q->k5_ss = q->kcaoff;
  q->b1 = q->k1m * q->MgADP;
  q->a2 = q->k2p;
  q->a4 = ((q->k4p * q->MgATP) / q->Kmgatp) / (1.00000 + q->MgATP / q->Kmgatp);
  q->Pnak = (ct == 1.0 ? q->Pnak_b * 0.900000 : ct == 2.0 ? q->Pnak_b * 0.700000 : q->Pnak_b);
}

static double hill_factor(double conc, double ic50, double h) {
  /* ___applyDrugEffect, Ohara_Rudy_2011.cpp:469-485 (epsilon 10E-14) */
  return (ic50 > 10E-14 && h > 10E-14) ? 1. / (1. + pow(conc / ic50, h)) : 1.;
}

/* quirks: 0 the intended forms; 1 the DrugSimulation build's quirks
 * (documented in cep_oracle.h); 2 the CEPCell_NEO build
 * (CEPCell_NEO/cellmodels/Ohara_Rudy_2011.cpp:456-520): celltype kept,
 * ___applyDutta on the intended constants (GKs, GKr, GK1, PCa, GNaL,
 * :456-463) but, like the Hill block (:505-520), after ___initConsts has
 * derived PCap, PCaNa and PCaK from PCa, which therefore stay unscaled. */
int cepo_ord_init(cepo_cell *c, double celltype, double conc, const double *ic50, int is_dutta,
                  int quirks) {
  ord_p *q = (ord_p *)c->p;
  memset(c->p, 0, sizeof(c->p));
  const int neo = quirks == 2;
  if (neo) quirks = 0;
  ord_base_consts(q, quirks ? 0.0 : celltype);
  if (is_dutta) {
    if (quirks) { /* ___applyDutta as written, Ohara_Rudy_2011.cpp:460-467 */
      q->Aff *= 1.870;
      q->GNaL *= 1.013;
      q->tjca *= 1.698;
      q->H *= 1.007;
      q->Gncx_b *= 2.661;
    } else {
      q->GKs *= 1.870;
      q->GKr *= 1.013;
      q->GK1 *= 1.698;
      q->PCa *= 1.007;
      if (!neo) derive_pca(q);
      q->GNaL *= 2.661;
    }
  }
  if (ic50) {
    q->PCa *= hill_factor(conc, ic50[0], ic50[1]);
    q->GK1 *= hill_factor(conc, ic50[2], ic50[3]);
    q->GKs *= hill_factor(conc, ic50[4], ic50[5]);
    q->GNa *= hill_factor(conc, ic50[6], ic50[7]);
    q->GNaL *= hill_factor(conc, ic50[8], ic50[9]);
    q->Gto *= hill_factor(conc, ic50[10], ic50[11]);
    q->GKr *= hill_factor(conc, ic50[12], ic50[13]);
    if (!quirks && !neo) derive_pca(q);
  }
  q->fcafp_dt = quirks ? 25.0 : 0.0;
  return 0;
}

void cepo_ord_set_pacing(cepo_cell *c, double bcl, double stim_start, double stim_dur,
                         double amp_scale) {
  /* CONSTANTS[BCL] = bcl_init; CONSTANTS[amp] *= stim_amp
   * (CEPCell_NEO/modules/cipa_drug_bench.cpp:146-147); negative start or
   * duration keep the model defaults. */
  ord_p *q = (ord_p *)c->p;
  q->BCL = bcl;
  if (stim_start >= 0) q->stim_start = stim_start;
  if (stim_dur >= 0) q->duration = stim_dur;
  q->amp *= amp_scale;
}

/* CONSTANTS[cumm_BCL], the start of the current pace of the cumulative
 * stimulus (tissue_stim == 2; CEPCell_NEO/cellmodels/Ohara_Rudy_2011.cpp:694-695). */
void cepo_ord_set_cumm(cepo_cell *c, double cumm_bcl) { ((ord_p *)c->p)->cumm_BCL = cumm_bcl; }

void cepo_ord_pacing(const cepo_cell *c, double *bcl, double *stim_start) {
  const ord_p *q = (const ord_p *)c->p;
  *bcl = q->BCL;
  *stim_start = q->stim_start;
}

/* Initial STATES of ___initConsts, Ohara_Rudy_2011.cpp:494-678. */
void cepo_ord_init_states(double *y) {
  for (int i = 0; i < ORD_NS; ++i) y[i] = 0.0;
  y[V] = -87; y[CaMKt] = 0; y[cass] = 1e-4; y[nai] = 7; y[nass] = 7; y[ki] = 145; y[kss] = 145;
  y[cansr] = 1.2; y[cajsr] = 1.2; y[cai] = 1e-4; y[m] = 0; y[hf] = 1; y[hs] = 1; y[j] = 1;
  y[hsp] = 1; y[jp] = 1; y[mL] = 0; y[hL] = 1; y[hLp] = 1; y[a] = 0; y[iF] = 1; y[iS] = 1;
  y[ap] = 0; y[iFp] = 1; y[iSp] = 1; y[d] = 0; y[ff] = 1; y[fs] = 1; y[fcaf] = 1; y[fcas] = 1;
  y[jca] = 1; y[ffp] = 1; y[fcafp] = 1; y[nca] = 0; y[xrf] = 0; y[xrs] = 0; y[xs1] = 0;
  y[xs2] = 0; y[xk1] = 1; y[Jrelnp] = 0; y[Jrelp] = 0;
}

/* Quantities computeRates produces that solveAnalytical consumes. */
typedef struct {
  double mss, tm, hss, thf, ths, jss, tj, hssp, thsp, tjp, mLss, tmL, hLss, hLssp, ass, ta, iss,
      tiF, tiS, assp, tiFp, tiSp, dss, td, fss, tff, tfs, fcass, tfcaf, tfcas, tffp, tfcafp, anca,
      km2n, xrss, txrf, txrs, xs1ss, txs1, xs2ss, txs2, xk1ss, txk1, Jrel_inf, tau_rel, Jrel_infp,
      tau_relp;
} ord_gates;

/* computeRates, Ohara_Rudy_2011.cpp:742-989 (same expression order). */
static void ord_compute(const cepo_cell *c, double TIME, const double *S, double *R_,
                        ord_gates *g, cepo_currents *cur) {
  const ord_p *q = (const ord_p *)c->p;
  const double v = S[V];
  double Istim;
  if (c->tissue_stim == 2)  /* hrv: the pace starts at cumm_BCL (:694-695) */
    Istim = (q->stim_start + q->cumm_BCL <= TIME && TIME < q->stim_start + q->cumm_BCL + q->duration ? q->amp : 0.0);
  else if (c->tissue_stim)
    Istim = c->is_s1 ? q->amp : 0.0;
  else
    Istim = (TIME >= q->stim_start && (TIME - q->stim_start) -
                                              floor((TIME - q->stim_start) / q->BCL) * q->BCL <=
                                          q->duration
                 ? q->amp
                 : 0.000000);
  g->hLss = 1.00000 / (1.00000 + exp((v + 87.6100) / 7.48800));
  g->hLssp = 1.00000 / (1.00000 + exp((v + 93.8100) / 7.48800));
  g->mss = 1.00000 / (1.00000 + exp(-(v + q->mssV1) / q->mssV2));
  g->tm = 1.00000 / (q->mtD1 * exp((v + q->mtV1) / q->mtV2) + q->mtD2 * exp(-(v + q->mtV3) / q->mtV4));
  g->hss = 1.00000 / (1.00000 + exp((v + q->hssV1) / q->hssV2));
  g->thf = 1.00000 / (1.43200e-05 * exp(-(v + 1.19600) / 6.28500) + 6.14900 * exp((v + 0.509600) / 20.2700));
  g->ths = 1.00000 / (0.00979400 * exp(-(v + 17.9500) / 28.0500) + 0.334300 * exp((v + 5.73000) / 56.6600));
  g->ass = 1.00000 / (1.00000 + exp(-(v - 14.3400) / 14.8200));
  g->ta = 1.05150 / (1.00000 / (1.20890 * (1.00000 + exp(-(v - 18.4099) / 29.3814))) +
                     3.50000 / (1.00000 + exp((v + 100.000) / 29.3814)));
  g->dss = 1.00000 / (1.00000 + exp(-(v + 3.94000) / 4.23000));
  g->td = 0.600000 + 1.00000 / (exp(-0.0500000 * (v + 6.00000)) + exp(0.0900000 * (v + 14.0000)));
  g->fss = 1.00000 / (1.00000 + exp((v + 19.5800) / 3.69600));
  g->tff = 7.00000 + 1.00000 / (0.00450000 * exp(-(v + 20.0000) / 10.0000) + 0.00450000 * exp((v + 20.0000) / 10.0000));
  g->tfs = 1000.00 + 1.00000 / (3.50000e-05 * exp(-(v + 5.00000) / 4.00000) + 3.50000e-05 * exp((v + 5.00000) / 6.00000));
  g->fcass = g->fss;
  g->km2n = S[jca] * 1.00000;
  g->anca = 1.00000 / (q->k2n / g->km2n + pow(1.00000 + q->Kmn / S[cass], 4.00000));
  g->xrss = 1.00000 / (1.00000 + exp(-(v + 8.33700) / 6.78900));
  g->txrf = 12.9800 + 1.00000 / (0.365200 * exp((v - 31.6600) / 3.86900) + 4.12300e-05 * exp(-(v - 47.7800) / 20.3800));
  g->txrs = 1.86500 + 1.00000 / (0.0662900 * exp((v - 34.7000) / 7.35500) + 1.12800e-05 * exp(-(v - 29.7400) / 25.9400));
  g->xs1ss = 1.00000 / (1.00000 + exp(-(v + 11.6000) / 8.93200));
  g->txs1 = 817.300 + 1.00000 / (0.000232600 * exp((v + 48.2800) / 17.8000) + 0.00129200 * exp(-(v + 210.000) / 230.000));
  g->xk1ss = 1.00000 / (1.00000 + exp(-(v + 2.55380 * q->ko + 144.590) / (1.56920 * q->ko + 3.81150)));
  g->txk1 = 122.200 / (exp(-(v + 127.200) / 20.3600) + exp((v + 236.800) / 69.3300));
  g->jss = g->hss;
  g->tj = 2.03800 + 1.00000 / (0.0213600 * exp(-(v + 100.600) / 8.28100) + 0.305200 * exp((v + 0.994100) / 38.4500));
  g->assp = 1.00000 / (1.00000 + exp(-(v - 24.3400) / 14.8200));
  g->tfcaf = 7.00000 + 1.00000 / (0.0400000 * exp(-(v - 4.00000) / 7.00000) + 0.0400000 * exp((v - 4.00000) / 7.00000));
  g->tfcas = 100.000 + 1.00000 / (0.000120000 * exp(-v / 3.00000) + 0.000120000 * exp(v / 7.00000));
  g->tffp = 2.50000 * g->tff;
  g->xs2ss = g->xs1ss;
  g->txs2 = 1.00000 / (0.0100000 * exp((v - 50.0000) / 20.0000) + 0.0193000 * exp(-(v + 66.5400) / 31.0000));
  const double CaMKb = (q->CaMKo * (1.00000 - S[CaMKt])) / (1.00000 + q->KmCaM / S[cass]);
  g->hssp = 1.00000 / (1.00000 + exp((v + 89.1000) / 6.08600));
  g->thsp = 3.00000 * g->ths;
  g->tjp = 1.46000 * g->tj;
  g->mLss = 1.00000 / (1.00000 + exp(-(v + 42.8500) / 5.26400));
  g->tmL = g->tm;
  g->tfcafp = 2.50000 * g->tfcaf;
  g->iss = 1.00000 / (1.00000 + exp((v + 43.9400) / 5.71100));
  const double delta_epi = (q->celltype == 1.0 ? 1.00000 - 0.950000 / (1.00000 + exp((v + 70.0000) / 5.00000)) : 1.00000);
  const double tiF_b = 4.56200 + 1.00000 / (0.393300 * exp(-(v + 100.000) / 100.000) + 0.0800400 * exp((v + 50.0000) / 16.5900));
  g->tiF = tiF_b * delta_epi;
  const double tiS_b = 23.6200 + 1.00000 / (0.00141600 * exp(-(v + 96.5200) / 59.0500) + 1.78000e-08 * exp((v + 114.100) / 8.07900));
  g->tiS = tiS_b * delta_epi;
  const double dti_develop = 1.35400 + 0.000100000 / (exp((v - 167.400) / 15.8900) + exp(-(v - 12.2300) / 0.215400));
  const double dti_recover = 1.00000 - 0.500000 / (1.00000 + exp((v + 70.0000) / 20.0000));
  g->tiFp = dti_develop * dti_recover * g->tiF;
  g->tiSp = dti_develop * dti_recover * g->tiS;
  const double f = q->Aff * S[ff] + q->Afs * S[fs];
  const double Afcaf = 0.300000 + 0.600000 / (1.00000 + exp((v - 10.0000) / 10.0000));
  const double Afcas = 1.00000 - Afcaf;
  const double fca = Afcaf * S[fcaf] + Afcas * S[fcas];
  const double fp = q->Aff * S[ffp] + q->Afs * S[fs];
  const double fcap = Afcaf * S[fcafp] + Afcas * S[fcas];
  const double vffrt = (v * q->F * q->F) / (q->R * q->T);
  const double vfrt = (v * q->F) / (q->R * q->T);
  const double PhiCaL = (4.00000 * vffrt * (S[cass] * exp(2.00000 * vfrt) - 0.341000 * q->cao)) / (exp(2.00000 * vfrt) - 1.00000);
  const double CaMKa = CaMKb + S[CaMKt];
  const double fICaLp = 1.00000 / (1.00000 + q->KmCaMK / CaMKa);
  const double ICaL = (1.00000 - fICaLp) * q->PCa * PhiCaL * S[d] * (f * (1.00000 - S[nca]) + S[jca] * fca * S[nca]) +
                      fICaLp * q->PCap * PhiCaL * S[d] * (fp * (1.00000 - S[nca]) + S[jca] * fcap * S[nca]);
  const double Jrel_inf_temp = (q->a_rel * -ICaL) / (1.00000 + 1.00000 * pow(1.50000 / S[cajsr], 8.00000));
  g->Jrel_inf = (q->celltype == 2.0 ? Jrel_inf_temp * 1.70000 : Jrel_inf_temp);
  const double tau_rel_temp = q->bt / (1.00000 + 0.0123000 / S[cajsr]);
  g->tau_rel = (tau_rel_temp < 0.00100000 ? 0.00100000 : tau_rel_temp);
  const double Jrel_temp = (q->a_relp * -ICaL) / (1.00000 + pow(1.50000 / S[cajsr], 8.00000));
  g->Jrel_infp = (q->celltype == 2.0 ? Jrel_temp * 1.70000 : Jrel_temp);
  const double tau_relp_temp = q->btp / (1.00000 + 0.0123000 / S[cajsr]);
  g->tau_relp = (tau_relp_temp < 0.00100000 ? 0.00100000 : tau_relp_temp);
  const double EK = ((q->R * q->T) / q->F) * log(q->ko / S[ki]);
  const double AiF = 1.00000 / (1.00000 + exp((v - 213.600) / 151.200));
  const double AiS = 1.00000 - AiF;
  const double i_ = AiF * S[iF] + AiS * S[iS];
  const double ip = AiF * S[iFp] + AiS * S[iSp];
  const double fItop = 1.00000 / (1.00000 + q->KmCaMK / CaMKa);
  const double Ito = q->Gto * (v - EK) * ((1.00000 - fItop) * S[a] * i_ + fItop * S[ap] * ip);
  const double Axrf = 1.00000 / (1.00000 + exp((v + 54.8100) / 38.2100));
  const double Axrs = 1.00000 - Axrf;
  const double xr = Axrf * S[xrf] + Axrs * S[xrs];
  const double rkr = ((1.00000 / (1.00000 + exp((v + 55.0000) / 75.0000))) * 1.00000) / (1.00000 + exp((v - 10.0000) / 30.0000));
  const double IKr = q->GKr * pow((q->ko / 5.40000), 1.0 / 2) * xr * rkr * (v - EK);
  const double EKs = ((q->R * q->T) / q->F) * log((q->ko + q->PKNa * q->nao) / (S[ki] + q->PKNa * S[nai]));
  const double KsCa = 1.00000 + 0.600000 / (1.00000 + pow(3.80000e-05 / S[cai], 1.40000));
  const double IKs = q->GKs * KsCa * S[xs1] * S[xs2] * (v - EKs);
  const double rk1 = 1.00000 / (1.00000 + exp(((v + 105.800) - 2.60000 * q->ko) / 9.49300));
  const double IK1 = q->GK1 * pow(q->ko, 1.0 / 2) * rk1 * S[xk1] * (v - EK);
  const double Knao = q->Knao0 * exp(((1.00000 - q->delta) * v * q->F) / (3.00000 * q->R * q->T));
  const double a3 = (q->k3p * pow(q->ko / q->Kko, 2.00000)) / ((pow(1.00000 + q->nao / Knao, 3.00000) + pow(1.00000 + q->ko / q->Kko, 2.00000)) - 1.00000);
  const double P = q->eP / (1.00000 + q->H / q->Khp + S[nai] / q->Knap + S[ki] / q->Kxkur);
  const double b3 = (q->k3m * P * q->H) / (1.00000 + q->MgATP / q->Kmgatp);
  const double Knai = q->Knai0 * exp((q->delta * v * q->F) / (3.00000 * q->R * q->T));
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
  const double xkb = 1.00000 / (1.00000 + exp(-(v - 14.4800) / 18.3400));
  const double IKb = q->GKb * xkb * (v - EK);
  const double JdiffK = (S[kss] - S[ki]) / 2.00000;
  const double PhiCaK = (1.00000 * vffrt * (0.750000 * S[kss] * exp(1.00000 * vfrt) - 0.750000 * q->ko)) / (exp(1.00000 * vfrt) - 1.00000);
  const double ICaK = (1.00000 - fICaLp) * q->PCaK * PhiCaK * S[d] * (f * (1.00000 - S[nca]) + S[jca] * fca * S[nca]) +
                      fICaLp * q->PCaKp * PhiCaK * S[d] * (fp * (1.00000 - S[nca]) + S[jca] * fcap * S[nca]);
  const double ENa = ((q->R * q->T) / q->F) * log(q->nao / S[nai]);
  const double h_ = q->Ahf * S[hf] + q->Ahs * S[hs];
  const double hp = q->Ahf * S[hf] + q->Ahs * S[hsp];
  const double fINap = 1.00000 / (1.00000 + q->KmCaMK / CaMKa);
  const double INa = q->GNa * (v - ENa) * pow(S[m], 3.00000) * ((1.00000 - fINap) * h_ * S[j] + fINap * hp * S[jp]);
  const double fINaLp = 1.00000 / (1.00000 + q->KmCaMK / CaMKa);
  const double INaL = q->GNaL * (v - ENa) * S[mL] * ((1.00000 - fINaLp) * S[hL] + fINaLp * S[hLp]);
  const double allo_i = 1.00000 / (1.00000 + pow(q->KmCaAct / S[cai], 2.00000));
  const double hna = exp((q->qna * v * q->F) / (q->R * q->T));
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
  const double hca = exp((q->qca * v * q->F) / (q->R * q->T));
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
  const double INaCa_i = 0.800000 * q->Gncx * allo_i * (q->zna * JncxNa_i + q->zca * JncxCa_i);
  const double INab = (q->PNab * vffrt * (S[nai] * exp(vfrt) - q->nao)) / (exp(vfrt) - 1.00000);
  const double JdiffNa = (S[nass] - S[nai]) / 2.00000;
  const double PhiCaNa = (1.00000 * vffrt * (0.750000 * S[nass] * exp(1.00000 * vfrt) - 0.750000 * q->nao)) / (exp(1.00000 * vfrt) - 1.00000);
  const double ICaNa = (1.00000 - fICaLp) * q->PCaNa * PhiCaNa * S[d] * (f * (1.00000 - S[nca]) + S[jca] * fca * S[nca]) +
                       fICaLp * q->PCaNap * PhiCaNa * S[d] * (fp * (1.00000 - S[nca]) + S[jca] * fcap * S[nca]);
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
  const double INaCa_ss = 0.200000 * q->Gncx * allo_ss * (q->zna * JncxNa_ss + q->zca * JncxCa_ss);
  const double IpCa = (q->GpCa * S[cai]) / (q->KmCap + S[cai]);
  const double ICab = (q->PCab * 4.00000 * vffrt * (S[cai] * exp(2.00000 * vfrt) - 0.341000 * q->cao)) / (exp(2.00000 * vfrt) - 1.00000);
  const double Jdiff = (S[cass] - S[cai]) / 0.200000;
  const double fJrelp = 1.00000 / (1.00000 + q->KmCaMK / CaMKa);
  const double Jrel = (1.00000 - fJrelp) * S[Jrelnp] + fJrelp * S[Jrelp];
  const double Bcass = 1.00000 / (1.00000 + (q->BSRmax * q->KmBSR) / pow(q->KmBSR + S[cass], 2.00000) +
                                  (q->BSLmax * q->KmBSL) / pow(q->KmBSL + S[cass], 2.00000));
  const double Jupnp = (q->upScale * 0.00437500 * S[cai]) / (S[cai] + 0.000920000);
  const double Jupp = (q->upScale * 2.75000 * 0.00437500 * S[cai]) / ((S[cai] + 0.000920000) - 0.000170000);
  const double fJupp = 1.00000 / (1.00000 + q->KmCaMK / CaMKa);
  const double Jleak = (0.00393750 * S[cansr]) / 15.0000;
  const double Jup = ((1.00000 - fJupp) * Jupnp + fJupp * Jupp) - Jleak;
  const double Bcai = 1.00000 / (1.00000 + (q->cmdnmax * q->kmcmdn) / pow(q->kmcmdn + S[cai], 2.00000) +
                                 (q->trpnmax * q->kmtrpn) / pow(q->kmtrpn + S[cai], 2.00000));
  const double Jtr = (S[cansr] - S[cajsr]) / 100.000;
  const double Bcajsr = 1.00000 / (1.00000 + (q->csqnmax * q->kmcsqn) / pow(q->kmcsqn + S[cajsr], 2.00000));

  if (R_) {
    R_[hL] = (g->hLss - S[hL]) / q->thL;
    R_[hLp] = (g->hLssp - S[hLp]) / q->thLp;
    R_[m] = (g->mss - S[m]) / g->tm;
    R_[hf] = (g->hss - S[hf]) / g->thf;
    R_[hs] = (g->hss - S[hs]) / g->ths;
    R_[a] = (g->ass - S[a]) / g->ta;
    R_[d] = (g->dss - S[d]) / g->td;
    R_[ff] = (g->fss - S[ff]) / g->tff;
    R_[fs] = (g->fss - S[fs]) / g->tfs;
    R_[jca] = (g->fcass - S[jca]) / q->tjca;
    R_[nca] = g->anca * q->k2n - S[nca] * g->km2n;
    R_[xrf] = (g->xrss - S[xrf]) / g->txrf;
    R_[xrs] = (g->xrss - S[xrs]) / g->txrs;
    R_[xs1] = (g->xs1ss - S[xs1]) / g->txs1;
    R_[xk1] = (g->xk1ss - S[xk1]) / g->txk1;
    R_[j] = (g->jss - S[j]) / g->tj;
    R_[ap] = (g->assp - S[ap]) / g->ta;
    R_[fcaf] = (g->fcass - S[fcaf]) / g->tfcaf;
    R_[fcas] = (g->fcass - S[fcas]) / g->tfcas;
    R_[ffp] = (g->fss - S[ffp]) / g->tffp;
    R_[xs2] = (g->xs2ss - S[xs2]) / g->txs2;
    R_[CaMKt] = q->aCaMK * CaMKb * (CaMKb + S[CaMKt]) - q->bCaMK * S[CaMKt];
    R_[hsp] = (g->hssp - S[hsp]) / g->thsp;
    R_[jp] = (g->jss - S[jp]) / g->tjp;
    R_[mL] = (g->mLss - S[mL]) / g->tmL;
    R_[fcafp] = (g->fcass - S[fcafp]) / g->tfcafp;
    R_[iF] = (g->iss - S[iF]) / g->tiF;
    R_[iS] = (g->iss - S[iS]) / g->tiS;
    R_[iFp] = (g->iss - S[iFp]) / g->tiFp;
    R_[iSp] = (g->iss - S[iSp]) / g->tiSp;
    R_[Jrelnp] = (g->Jrel_inf - S[Jrelnp]) / g->tau_rel;
    R_[Jrelp] = (g->Jrel_infp - S[Jrelp]) / g->tau_relp;
    R_[ki] = (-((Ito + IKr + IKs + IK1 + IKb + Istim) - 2.00000 * INaK) * q->cm * q->Acap) / (q->F * q->vmyo) +
             (JdiffK * q->vss) / q->vmyo;
    R_[kss] = (-ICaK * q->cm * q->Acap) / (q->F * q->vss) - JdiffK;
    R_[nai] = (-(INa + INaL + 3.00000 * INaCa_i + 3.00000 * INaK + INab) * q->Acap * q->cm) / (q->F * q->vmyo) +
              (JdiffNa * q->vss) / q->vmyo;
    R_[nass] = (-(ICaNa + 3.00000 * INaCa_ss) * q->cm * q->Acap) / (q->F * q->vss) - JdiffNa;
    R_[V] = -(INa + INaL + Ito + ICaL + ICaNa + ICaK + IKr + IKs + IK1 + INaCa_i + INaCa_ss + INaK + INab + IKb +
              IpCa + ICab + Istim);
    R_[cass] = Bcass * (((-(ICaL - 2.00000 * INaCa_ss) * q->cm * q->Acap) / (2.00000 * q->F * q->vss) +
                         (Jrel * q->vjsr) / q->vss) - Jdiff);
    R_[cai] = Bcai * (((-((IpCa + ICab) - 2.00000 * INaCa_i) * q->cm * q->Acap) / (2.00000 * q->F * q->vmyo) -
                       (Jup * q->vnsr) / q->vmyo) + (Jdiff * q->vss) / q->vmyo);
    R_[cansr] = Jup - (Jtr * q->vjsr) / q->vnsr;
    R_[cajsr] = Bcajsr * (Jtr - Jrel);
  }
  if (cur) {
    cur->INa = INa; cur->INaL = INaL; cur->Ito = Ito; cur->ICaL = ICaL; cur->IKr = IKr;
    cur->IKs = IKs; cur->IK1 = IK1;
    cur->dVdt = R_ ? R_[V] : 0.0;
  }
}

void cepo_ord_rates(const cepo_cell *c, double t, const double *y, double *dydt, cepo_currents *cur) {
  double r[ORD_NS];
  ord_gates g;
  ord_compute(c, t, y, dydt ? dydt : r, &g, cur);
}

/* computeRates then solveAnalytical (non-EULER branch,
 * Ohara_Rudy_2011.cpp:1036-1094). */
void cepo_ord_step(const cepo_cell *c, double t, double dt, double *S, cepo_currents *cur) {
  const ord_p *q = (const ord_p *)c->p;
  double R_[ORD_NS];
  ord_gates g;
  ord_compute(c, t, S, R_, &g, cur);
  const double dfca = q->fcafp_dt != 0.0 ? q->fcafp_dt : dt;
  S[m] = g.mss - (g.mss - S[m]) * exp(-dt / g.tm);
  S[hf] = g.hss - (g.hss - S[hf]) * exp(-dt / g.thf);
  S[hs] = g.hss - (g.hss - S[hs]) * exp(-dt / g.ths);
  S[j] = g.jss - (g.jss - S[j]) * exp(-dt / g.tj);
  S[hsp] = g.hssp - (g.hssp - S[hsp]) * exp(-dt / g.thsp);
  S[jp] = g.jss - (g.jss - S[jp]) * exp(-dt / g.tjp);
  S[mL] = g.mLss - (g.mLss - S[mL]) * exp(-dt / g.tmL);
  S[hL] = g.hLss - (g.hLss - S[hL]) * exp(-dt / q->thL);
  S[hLp] = g.hLssp - (g.hLssp - S[hLp]) * exp(-dt / q->thLp);
  S[a] = g.ass - (g.ass - S[a]) * exp(-dt / g.ta);
  S[iF] = g.iss - (g.iss - S[iF]) * exp(-dt / g.tiF);
  S[iS] = g.iss - (g.iss - S[iS]) * exp(-dt / g.tiS);
  S[ap] = g.assp - (g.assp - S[ap]) * exp(-dt / g.ta);
  S[iFp] = g.iss - (g.iss - S[iFp]) * exp(-dt / g.tiFp);
  S[iSp] = g.iss - (g.iss - S[iSp]) * exp(-dt / g.tiSp);
  S[d] = g.dss - (g.dss - S[d]) * exp(-dt / g.td);
  S[ff] = g.fss - (g.fss - S[ff]) * exp(-dt / g.tff);
  S[fs] = g.fss - (g.fss - S[fs]) * exp(-dt / g.tfs);
  S[fcaf] = g.fcass - (g.fcass - S[fcaf]) * exp(-dt / g.tfcaf);
  S[fcas] = g.fcass - (g.fcass - S[fcas]) * exp(-dt / g.tfcas);
  S[jca] = g.fcass - (g.fcass - S[jca]) * exp(-dt / q->tjca);
  S[ffp] = g.fss - (g.fss - S[ffp]) * exp(-dt / g.tffp);
  S[fcafp] = g.fcass - (g.fcass - S[fcafp]) * exp(-dfca / g.tfcafp);
  S[nca] = g.anca * q->k2n / g.km2n - (g.anca * q->k2n / g.km2n - S[nca]) * exp(-g.km2n * dt);
  S[xrf] = g.xrss - (g.xrss - S[xrf]) * exp(-dt / g.txrf);
  S[xrs] = g.xrss - (g.xrss - S[xrs]) * exp(-dt / g.txrs);
  S[xs1] = g.xs1ss - (g.xs1ss - S[xs1]) * exp(-dt / g.txs1);
  S[xs2] = g.xs2ss - (g.xs2ss - S[xs2]) * exp(-dt / g.txs2);
  S[xk1] = g.xk1ss - (g.xk1ss - S[xk1]) * exp(-dt / g.txk1);
  S[Jrelnp] = g.Jrel_inf - (g.Jrel_inf - S[Jrelnp]) * exp(-dt / g.tau_rel);
  S[Jrelp] = g.Jrel_infp - (g.Jrel_infp - S[Jrelp]) * exp(-dt / g.tau_relp);
  S[CaMKt] = S[CaMKt] + R_[CaMKt] * dt;
  S[V] = S[V] + R_[V] * dt;
  S[nai] = S[nai] + R_[nai] * dt;
  S[nass] = S[nass] + R_[nass] * dt;
  S[ki] = S[ki] + R_[ki] * dt;
  S[kss] = S[kss] + R_[kss] * dt;
  S[cai] = S[cai] + R_[cai] * dt;
  S[cass] = S[cass] + R_[cass] * dt;
  S[cansr] = S[cansr] + R_[cansr] * dt;
  S[cajsr] = S[cajsr] + R_[cajsr] * dt;
}

/* CONSTANTS[x] *= f after initConsts, x one of the CEP scale conductances
 * (0 GNa, 1 GNaL, 2 Gto, 3 PCa, 4 GKr, 5 GKs, 6 GK1, 11 GKb, 12 Gncx,
 * 13 Pnak), as the reference's call sites do (cipa_drug_bench.cpp:148).
 * Returns -1 for a conductance the model has no constant for here. */
int cepo_ord_scale(cepo_cell *c, int g, double f) {
  ord_p *q = (ord_p *)c->p;
  double *x = g == 0 ? &q->GNa : g == 1 ? &q->GNaL : g == 2 ? &q->Gto : g == 3 ? &q->PCa : g == 4 ? &q->GKr
            : g == 5 ? &q->GKs : g == 6 ? &q->GK1 : g == 11 ? &q->GKb : g == 12 ? &q->Gncx : g == 13 ? &q->Pnak : 0;
  if (!x) return -1;
  *x *= f;
  return 0;
}
