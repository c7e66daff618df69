/*
 * TEST INFRASTRUCTURE ONLY. CPU restatement of the CiPA-ORd v1 2017 model
 * (O'Hara-Rudy with the dynamic hERG Markov IKr and drug binding/trapping)
 * as CEPCell_NEO/cellmodels/ohara_rudy_cipa_v1_2017.cpp implements it:
 * ___initConsts (:1246-1501, the active block), initConsts(type, conc, hill)
 * (:1515-1539) and computeRates (:2156-2404, the active block). The RATES
 * keep the reference's evaluation order and are pinned bit for bit against
 * the reference compiled from its own sources (tests/test_oracle_pin.py).
 *
 * The reference integrates this model only with CVODE (its solveAnalytical
 * is empty). The fixed-step scheme here follows the reference's own ORd
 * scheme (Ohara_Rudy_2011.cpp:1036-1094): Rush-Larsen for the
 * Hodgkin-Huxley gates and forward Euler for V, ions, CaMKII and the nine
 * Markov IKr states. (A per-state Rush-Larsen form of the Markov chain was
 * tried and rejected: the stiff IC1 <-> C1 exchange makes it inaccurate,
 * APD90 off by tens of ms, while forward Euler stays within 0.25 ms of a
 * ten times finer step.)
 *
 * quirks = 1 reproduces the reference: ___initConsts resets CONSTANTS[0]
 * (celltype) to 0, the drug block scales PCa after PCap/PCaNa/PCaK/
 * PCaNap/PCaKp were derived from it, and a negative Vhalf is ignored.
 */
#include <math.h>
#include <string.h>
#include "cep_oracle.h"

typedef struct {
  double celltype, nao, cao, ko, R, T, F, zna, zca, zk, L, rad, stim_start, stim_end, amp, stim_period,
      duration;
  double KmCaMK, aCaMK, bCaMK, CaMKo, KmCaM, cmdnmax_b, kmcmdn, trpnmax, kmtrpn, BSRmax, KmBSR, BSLmax, KmBSL,
      csqnmax, kmcsqn, cm, PKNa, mssV1, mssV2, mtV1, mtV2, mtD1, mtD2, mtV3, mtV4, hssV1, hssV2, Ahf, GNa,
      shift_INa_inact, thL, GNaL_b, Gto_b, Kmn, k2n, PCa_b, GKr_b;
  double A1, B1, q1, A2, B2, q2, A3, B3, q3, A4, B4, q4, A11, B11, q11, A21, B21, q21, A31, B31, q31, A41, B41,
      q41, A51, B51, q51, A52, B52, q52, A53, B53, q53, A61, B61, q61, A62, B62, q62, A63, B63, q63;
  double Kmax, Ku, n, halfmax, Kt, Vhalf, Temp, GKs_b, txs1_max, GK1_b;
  double kna1, kna2, kna3, kasymm, wna, wca, wnaca, kcaon, kcaoff, qna, qca, KmCaAct, Gncx_b, k1p, k1m, k2p,
      k2m, k3p, k3m, k4p, k4m, Knai0, Knao0, delta, Kki, Kko, MgADP, MgATP, Kmgatp, H, eP, Khp, Knap, Kxkur,
      Pnak_b, GKb_b, PNab, PCab, GpCa, KmCap, bt, Jrel_scaling_factor, Jup_b;
  /* derived */
  double frt, cmdnmax, Ahs, thLp, GNaL, Gto, Aff, PCa, tjca, v0, GKr, GKs, GK1, vcell, GKb, v0_INab, v0_ICab,
      a_rel, btp, upScale, ffrt, Afs, PCap, PCaNa, PCaK, B_1, B_2, B_3, Ageo, B_INab, B_ICab, a_relp, PCaNap,
      PCaKp, Acap, vmyo, vnsr, vjsr, vss, h10_i, h11_i, h12_i, k1_i, k2_i, k5_i, Gncx, h10_ss, h11_ss, h12_ss,
      k1_ss, k2_ss, k5_ss, b1, a2, a4, Pnak;
  double D; /* drug concentration (STATES[D] in the reference) */
} cipa_p;

_Static_assert(sizeof(cipa_p) <= CEPO_MAX_PARAMS * sizeof(double), "cipa_p too large");

enum {
  V = 0, CaMKt, cass, nai, nass, ki, kss, cansr, cajsr, cai, m, hf, hs, j, hsp, jp, mL, hL, hLp, a, iF,
  iS, ap, iFp, iSp, d, ff, fs, fcaf, fcas, jca, ffp, fcafp, nca, IC1, IC2, C1, C2, O, IO, IObound, Obound,
  Cbound, Dst, xs1, xs2, xk1, Jrelnp, Jrelp, CIPA_NS
};

static void derive_pca(cipa_p *q) {
  q->PCap = 1.10000 * q->PCa;
  q->PCaNa = 0.00125000 * q->PCa;
  q->PCaK = 0.000357400 * q->PCa;
  q->PCaNap = 0.00125000 * q->PCap;
  q->PCaKp = 0.000357400 * q->PCap;
}

/* ___initConsts active block, ohara_rudy_cipa_v1_2017.cpp:1246-1501 */
static void cipa_base(cipa_p *q, double ct) {
  q->celltype = ct;
  q->nao = 140; q->cao = 1.8; q->ko = 5.4; q->R = 8314; q->T = 310; q->F = 96485; q->zna = 1; q->zca = 2;
  q->zk = 1; q->L = 0.01; q->rad = 0.0011; q->stim_start = 10; q->stim_end = 100000000000000000;
  q->amp = -80; q->stim_period = 1000; q->duration = 0.5; q->KmCaMK = 0.15; q->aCaMK = 0.05;
  q->bCaMK = 0.00068; q->CaMKo = 0.05; q->KmCaM = 0.0015; q->cmdnmax_b = 0.05; q->kmcmdn = 0.00238;
  q->trpnmax = 0.07; q->kmtrpn = 0.0005; q->BSRmax = 0.047; q->KmBSR = 0.00087; q->BSLmax = 1.124;
  q->KmBSL = 0.0087; q->csqnmax = 10; q->kmcsqn = 0.8; q->cm = 1; q->PKNa = 0.01833; q->mssV1 = 39.57;
  q->mssV2 = 9.871; q->mtV1 = 11.64; q->mtV2 = 34.77; q->mtD1 = 6.765; q->mtD2 = 8.552; q->mtV3 = 77.42;
  q->mtV4 = 5.955; q->hssV1 = 82.9; q->hssV2 = 6.086; q->Ahf = 0.99; q->GNa = 75; q->shift_INa_inact = 0;
  q->thL = 200; q->GNaL_b = 0.019957499999999975; q->Gto_b = 0.02; q->Kmn = 0.002; q->k2n = 1000;
  q->PCa_b = 0.0001007; q->GKr_b = 0.04658545454545456;
  q->A1 = 0.0264; q->B1 = 4.631E-05; q->q1 = 4.843; q->A2 = 4.986E-06; q->B2 = -0.004226; q->q2 = 4.23;
  q->A3 = 0.001214; q->B3 = 0.008516; q->q3 = 4.962; q->A4 = 1.854E-05; q->B4 = -0.04641; q->q4 = 3.769;
  q->A11 = 0.0007868; q->B11 = 1.535E-08; q->q11 = 4.942; q->A21 = 5.455E-06; q->B21 = -0.1688;
  q->q21 = 4.156; q->A31 = 0.005509; q->B31 = 7.771E-09; q->q31 = 4.22; q->A41 = 0.001416;
  q->B41 = -0.02877; q->q41 = 1.459; q->A51 = 0.4492; q->B51 = 0.008595; q->q51 = 5; q->A52 = 0.3181;
  q->B52 = 3.613E-08; q->q52 = 4.663; q->A53 = 0.149; q->B53 = 0.004668; q->q53 = 2.412; q->A61 = 0.01241;
  q->B61 = 0.1725; q->q61 = 5.568; q->A62 = 0.3226; q->B62 = -0.0006575; q->q62 = 5; q->A63 = 0.008978;
  q->B63 = -0.02215; q->q63 = 5.682;
  q->Kmax = 0; q->Ku = 0; q->n = 1; q->halfmax = 1; q->Kt = 0; q->Vhalf = 1; q->Temp = 37;
  q->GKs_b = 0.006358000000000001; q->txs1_max = 817.3; q->GK1_b = 0.3239783999999998;
  q->kna1 = 15; q->kna2 = 5; q->kna3 = 88.12; q->kasymm = 12.5; q->wna = 6e4; q->wca = 6e4; q->wnaca = 5e3;
  q->kcaon = 1.5e6; q->kcaoff = 5e3; q->qna = 0.5224; q->qca = 0.167; q->KmCaAct = 150e-6;
  q->Gncx_b = 0.0008; q->k1p = 949.5; q->k1m = 182.4; q->k2p = 687.2; q->k2m = 39.4; q->k3p = 1899;
  q->k3m = 79300; q->k4p = 639; q->k4m = 40; q->Knai0 = 9.073; q->Knao0 = 27.78; q->delta = -0.155;
  q->Kki = 0.5; q->Kko = 0.3582; q->MgADP = 0.05; q->MgATP = 9.8; q->Kmgatp = 1.698e-7; q->H = 1e-7;
  q->eP = 4.2; q->Khp = 1.698e-7; q->Knap = 224; q->Kxkur = 292; q->Pnak_b = 30; q->GKb_b = 0.003;
  q->PNab = 3.75e-10; q->PCab = 2.5e-8; q->GpCa = 0.0005; q->KmCap = 0.0005; q->bt = 4.75;
  q->Jrel_scaling_factor = 1.0; q->Jup_b = 1.0;
  q->frt = q->F / (q->R * q->T);
  q->cmdnmax = (ct == 1.0 ? q->cmdnmax_b * 1.30000 : q->cmdnmax_b);
  q->Ahs = 1.00000 - q->Ahf;
  q->thLp = 3.00000 * q->thL;
  q->GNaL = (ct == 1.0 ? q->GNaL_b * 0.600000 : q->GNaL_b);
  q->Gto = (ct == 1.0 ? q->Gto_b * 4.00000 : ct == 2.0 ? q->Gto_b * 4.00000 : q->Gto_b);
  q->Aff = 0.600000;
  q->PCa = (ct == 1.0 ? q->PCa_b * 1.20000 : ct == 2.0 ? q->PCa_b * 2.50000 : q->PCa_b);
  q->tjca = 75.0000;
  q->v0 = 0.000000;
  q->GKr = (ct == 1.0 ? q->GKr_b * 1.30000 : ct == 2.0 ? q->GKr_b * 0.800000 : q->GKr_b);
  q->GKs = (ct == 1.0 ? q->GKs_b * 1.40000 : q->GKs_b);
  q->GK1 = (ct == 1.0 ? q->GK1_b * 1.20000 : ct == 2.0 ? q->GK1_b * 1.30000 : q->GK1_b);
  q->vcell = 1000.00 * 3.14000 * q->rad * q->rad * q->L;
  q->GKb = (ct == 1.0 ? q->GKb_b * 0.600000 : q->GKb_b);
  q->v0_INab = 0.000000;
  q->v0_ICab = 0.000000;
  q->a_rel = 0.500000 * q->bt;
  q->btp = 1.25000 * q->bt;
  q->upScale = (ct == 1.0 ? 1.30000 : 1.00000);
  q->ffrt = q->F * q->frt;
  q->Afs = 1.00000 - q->Aff;
  derive_pca(q);
  q->B_1 = 2.00000 * q->frt;
  q->B_2 = q->frt;
  q->B_3 = q->frt;
  q->Ageo = 2.00000 * 3.14000 * q->rad * q->rad + 2.00000 * 3.14000 * q->rad * q->L;
  q->B_INab = q->frt;
  q->B_ICab = 2.00000 * q->frt;
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

/* initConsts(type, conc, hill), ohara_rudy_cipa_v1_2017.cpp:1515-1539;
 * hill[19] (Kt) is an extension: the reference leaves Kt at 0. */
int cepo_cipa_init(cepo_cell *c, double celltype, double conc, const double *hill, int is_dutta, int quirks) {
  (void)is_dutta;
  cipa_p *q = (cipa_p *)c->p;
  memset(c->p, 0, sizeof(c->p));
  cipa_base(q, quirks ? 0.0 : celltype);
  q->D = conc;
#define HB(k) ((hill[k] > 10E-14 && hill[k + 1] > 10E-14) ? pow(1. + pow(q->D / hill[k], hill[k + 1]), -1) : 1.)
  q->PCa *= HB(0);
  q->GK1 *= HB(2);
  q->GKs *= HB(4);
  q->GNa *= HB(6);
  q->GNaL *= HB(8);
  q->Gto *= HB(10);
  q->GKr *= HB(12);
#undef HB
  if (!quirks) derive_pca(q);
  q->Kmax = (hill[14] > 10E-14) ? hill[14] : q->Kmax;
  q->Ku = (hill[15] > 10E-14) ? hill[15] : q->Ku;
  q->n = (hill[16] > 10E-14) ? hill[16] : q->n;
  q->halfmax = (hill[17] > 10E-14) ? hill[17] : q->halfmax;
  /* quirk (5): the reference's guard `> 10E-14` drops every negative Vhalf
   * (:1538), and CiPA's fitted Vhalf values are negative; without quirks any
   * non-zero Vhalf is used */
  if (quirks)
    q->Vhalf = (hill[18] > 10E-14) ? hill[18] : q->Vhalf;
  else if (hill[18] != 0.0)
    q->Vhalf = hill[18];
  if (hill[19] > 10E-14) q->Kt = hill[19];
  return 0;
}

void cepo_cipa_set_pacing(cepo_cell *c, double bcl, double stim_start, double stim_dur, double amp_scale) {
  cipa_p *q = (cipa_p *)c->p;
  q->stim_period = bcl;
  if (stim_start >= 0) q->stim_start = stim_start;
  if (stim_dur >= 0) q->duration = stim_dur;
  q->amp *= amp_scale;
}

void cepo_cipa_pacing(const cepo_cell *c, double *bcl, double *stim_start) {
  const cipa_p *q = (const cipa_p *)c->p;
  *bcl = q->stim_period;
  *stim_start = q->stim_start;
}

/* initial STATES of the active ___initConsts block; STATES[D] = conc as
 * initConsts(type, conc, hill) sets it (:1518) */
void cepo_cipa_init_states(const cepo_cell *c, double *y) {
  static const double y0[CIPA_NS] = {
      -88.00190465, 0.0125840447, 8.49e-05, 7.268004498, 7.268089977, 144.6555918, 144.6555651, 1.619574538,
      1.571234014, 8.6e-05, 0.007344121102, 0.6981071913, 0.6980895801, 0.6979908432, 0.4549485525,
      0.6979245865, 0.0001882617273, 0.5008548855, 0.2693065357, 0.001001097687, 0.9995541745, 0.5865061736,
      0.0005100862934, 0.9995541823, 0.6393399482, 2.34e-9, 0.9999999909, 0.9102412777, 0.9999999909,
      0.9998046777, 0.9999738312, 0.9999999909, 0.9999999909, 0.002749414044, 0.999637, 6.83208e-05,
      1.80145e-08, 8.26619e-05, 0.00015551, 5.67623e-05, 0, 0, 0, 0, 0.2707758025, 0.0001928503426,
      0.9967597594, 2.5e-7, 3.12e-7};
  memcpy(y, y0, sizeof(y0));
  y[Dst] = ((const cipa_p *)c->p)->D;
}

typedef struct {
  double mss, tm, hss, thf, ths, jss, tj, hssp, thsp, tjp, mLss, tmL, hLss, hLssp, ass, ta, iss, tiF, tiS,
      assp, tiFp, tiSp, dss, td, fss, tff, tfs, fcass, tfcaf, tfcas, tffp, tfcafp, anca, km2n, xs1ss, txs1,
      xs2ss, txs2, xk1ss, txk1, Jrel_inf, tau_rel, Jrel_infp, tau_relp;
  /* Markov IKr: A*exp(B*V) of every transition (Q10 applied separately, as
   * the reference orders the products), binding terms, largest outflow */
  double e11, e21, e51, e61, e3, e4, e52, e62, e1, e2, e31, e41, e53, e63, bind, unb, trap, lam_max;
} cipa_gates;

/* Q10 factor exp(((Temp - 20) * log(q)) / 10) as the reference forms it */
#define Q10(qq) exp(((q->Temp - 20.0000) * log(qq)) / 10.0000)

/* computeRates active block, ohara_rudy_cipa_v1_2017.cpp:2156-2404 */
static void cipa_compute(const cepo_cell *c, double TIME, const double *S, double *R_, cipa_gates *g,
                         cepo_currents *cur) {
  const cipa_p *q = (const cipa_p *)c->p;
  const double v = S[V];
  /* Markov IKr transition terms k_xy = A*exp(B*V)*state*Q10 (:2157-2165) */
  const double D = S[Dst];
  const double t11 = q->A11 * exp(q->B11 * v) * S[IC1] * Q10(q->q11);
  const double t21 = q->A21 * exp(q->B21 * v) * S[IC2] * Q10(q->q21);
  const double t51 = q->A51 * exp(q->B51 * v) * S[C1] * Q10(q->q51);
  const double t61 = q->A61 * exp(q->B61 * v) * S[IC1] * Q10(q->q61);
  const double t3 = q->A3 * exp(q->B3 * v) * S[IC2] * Q10(q->q3);
  const double t4 = q->A4 * exp(q->B4 * v) * S[IO] * Q10(q->q4);
  const double t52 = q->A52 * exp(q->B52 * v) * S[C2] * Q10(q->q52);
  const double t62 = q->A62 * exp(q->B62 * v) * S[IC2] * Q10(q->q62);
  const double t1 = q->A1 * exp(q->B1 * v) * S[C1] * Q10(q->q1);
  const double t2 = q->A2 * exp(q->B2 * v) * S[C2] * Q10(q->q2);
  const double t51b = q->A51 * exp(q->B51 * v) * S[C1] * Q10(q->q51);
  const double t61b = q->A61 * exp(q->B61 * v) * S[IC1] * Q10(q->q61);
  const double t31 = q->A31 * exp(q->B31 * v) * S[C2] * Q10(q->q31);
  const double t41 = q->A41 * exp(q->B41 * v) * S[O] * Q10(q->q41);
  const double t53 = q->A53 * exp(q->B53 * v) * S[O] * Q10(q->q53);
  const double t63 = q->A63 * exp(q->B63 * v) * S[IO] * Q10(q->q63);
  const double bind = (q->Kmax * q->Ku * exp(q->n * log(D))) / (exp(q->n * log(D)) + q->halfmax);
  g->e11 = q->A11 * exp(q->B11 * v); g->e21 = q->A21 * exp(q->B21 * v); g->e51 = q->A51 * exp(q->B51 * v);
  g->e61 = q->A61 * exp(q->B61 * v); g->e3 = q->A3 * exp(q->B3 * v); g->e4 = q->A4 * exp(q->B4 * v);
  g->e52 = q->A52 * exp(q->B52 * v); g->e62 = q->A62 * exp(q->B62 * v); g->e1 = q->A1 * exp(q->B1 * v);
  g->e2 = q->A2 * exp(q->B2 * v); g->e31 = q->A31 * exp(q->B31 * v); g->e41 = q->A41 * exp(q->B41 * v);
  g->e53 = q->A53 * exp(q->B53 * v); g->e63 = q->A63 * exp(q->B63 * v);
  const double unbind_io = (q->Ku * q->A53 * exp(q->B53 * v) * Q10(q->q53)) /
                           (q->A63 * exp(q->B63 * v) * Q10(q->q63));
  const double trap = q->Kt / (1.00000 + exp(-(v - q->Vhalf) / 6.78900));
  g->bind = bind; g->unb = unbind_io; g->trap = trap;
  {
    /* largest total outflow rate of a Markov state (1/ms) */
    const double o[9] = {g->e11 * Q10(q->q11) + g->e61 * Q10(q->q61),
                         g->e21 * Q10(q->q21) + g->e3 * Q10(q->q3) + g->e62 * Q10(q->q62),
                         g->e1 * Q10(q->q1) + g->e51 * Q10(q->q51),
                         g->e2 * Q10(q->q2) + g->e31 * Q10(q->q31) + g->e52 * Q10(q->q52),
                         g->e41 * Q10(q->q41) + g->e53 * Q10(q->q53) + bind,
                         g->e4 * Q10(q->q4) + g->e63 * Q10(q->q63) + bind,
                         unbind_io + q->Kt, q->Ku + q->Kt, 2.0 * trap};
    double mx = 0.0;
    for (int k = 0; k < 9; ++k) mx = o[k] > mx ? o[k] : mx;
    g->lam_max = mx;
  }
  if (R_) {
    R_[Dst] = 0.0;
    R_[IC1] = (-(t11 - t21) + t51) - t61;
    R_[IC2] = (((t11 - t21) - (t3 - t4)) + t52) - t62;
    R_[C1] = -(t1 - t2) - (t51b - t61b);
    R_[C2] = ((t1 - t2) - (t31 - t41)) - (t52 - t62);
    R_[O] = ((t31 - t41) - (t53 - t63)) - (bind * S[O] - q->Ku * S[Obound]);
    R_[IO] = ((t3 - t4) + t53 - t63) - (bind * S[IO] - unbind_io * S[IObound]);
    R_[IObound] = ((bind * S[IO] - unbind_io * S[IObound]) + trap * S[Cbound]) - q->Kt * S[IObound];
    R_[Obound] = ((bind * S[O] - q->Ku * S[Obound]) + trap * S[Cbound]) - q->Kt * S[Obound];
    R_[Cbound] = -(trap * S[Cbound] - q->Kt * S[Obound]) - (trap * S[Cbound] - q->Kt * S[IObound]);
  }
  g->hLss = 1.00000 / (1.00000 + exp((v + 87.6100) / 7.48800));
  g->hLssp = 1.00000 / (1.00000 + exp((v + 93.8100) / 7.48800));
  g->mss = 1.00000 / (1.00000 + exp(-(v + q->mssV1) / q->mssV2));
  g->tm = 1.00000 / (q->mtD1 * exp((v + q->mtV1) / q->mtV2) + q->mtD2 * exp(-(v + q->mtV3) / q->mtV4));
  g->hss = 1.00000 / (1.00000 + exp(((v + q->hssV1) - q->shift_INa_inact) / q->hssV2));
  g->thf = 1.00000 / (1.43200e-05 * exp(-((v + 1.19600) - q->shift_INa_inact) / 6.28500) +
                      6.14900 * exp(((v + 0.509600) - q->shift_INa_inact) / 20.2700));
  g->ths = 1.00000 / (0.00979400 * exp(-((v + 17.9500) - q->shift_INa_inact) / 28.0500) +
                      0.334300 * exp(((v + 5.73000) - q->shift_INa_inact) / 56.6600));
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
  g->xs1ss = 1.00000 / (1.00000 + exp(-(v + 11.6000) / 8.93200));
  g->txs1 = q->txs1_max + 1.00000 / (0.000232600 * exp((v + 48.2800) / 17.8000) + 0.00129200 * exp(-(v + 210.000) / 230.000));
  g->xk1ss = 1.00000 / (1.00000 + exp(-(v + 2.55380 * q->ko + 144.590) / (1.56920 * q->ko + 3.81150)));
  g->txk1 = 122.200 / (exp(-(v + 127.200) / 20.3600) + exp((v + 236.800) / 69.3300));
  const double CaMKb = (q->CaMKo * (1.00000 - S[CaMKt])) / (1.00000 + q->KmCaM / S[cass]);
  g->jss = g->hss;
  g->tj = 2.03800 + 1.00000 / (0.0213600 * exp(-((v + 100.600) - q->shift_INa_inact) / 8.28100) +
                               0.305200 * exp(((v + 0.994100) - q->shift_INa_inact) / 38.4500));
  g->assp = 1.00000 / (1.00000 + exp(-(v - 24.3400) / 14.8200));
  g->tfcaf = 7.00000 + 1.00000 / (0.0400000 * exp(-(v - 4.00000) / 7.00000) + 0.0400000 * exp((v - 4.00000) / 7.00000));
  g->tfcas = 100.000 + 1.00000 / (0.000120000 * exp(-v / 3.00000) + 0.000120000 * exp(v / 7.00000));
  g->tffp = 2.50000 * g->tff;
  g->xs2ss = g->xs1ss;
  g->txs2 = 1.00000 / (0.0100000 * exp((v - 50.0000) / 20.0000) + 0.0193000 * exp(-(v + 66.5400) / 31.0000));
  g->hssp = 1.00000 / (1.00000 + exp(((v + 89.1000) - q->shift_INa_inact) / 6.08600));
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
  const double vfrt = v * q->frt;
  const double A_1 = (4.00000 * q->ffrt * (S[cass] * exp(2.00000 * vfrt) - 0.341000 * q->cao)) / q->B_1;
  const double U_1 = q->B_1 * (v - q->v0);
  const double PhiCaL = (-1.00000e-07 <= U_1 && U_1 <= 1.00000e-07 ? A_1 * (1.00000 - 0.500000 * U_1)
                                                                   : (A_1 * U_1) / (exp(U_1) - 1.00000));
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
  const double IKr = q->GKr * pow((q->ko / 5.40000), 1.0 / 2) * S[O] * (v - EK);
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
  double Istim = (TIME >= q->stim_start && TIME <= q->stim_end &&
                          (TIME - q->stim_start) - floor((TIME - q->stim_start) / q->stim_period) * q->stim_period <=
                              q->duration
                      ? q->amp
                      : 0.000000);
  if (c->tissue_stim) Istim = c->is_s1 ? q->amp : 0.0;
  const double JdiffK = (S[kss] - S[ki]) / 2.00000;
  const double A_3 = (0.750000 * q->ffrt * (S[kss] * exp(vfrt) - q->ko)) / q->B_3;
  const double U_3 = q->B_3 * (v - q->v0);
  const double PhiCaK = (-1.00000e-07 <= U_3 && U_3 <= 1.00000e-07 ? A_3 * (1.00000 - 0.500000 * U_3)
                                                                   : (A_3 * U_3) / (exp(U_3) - 1.00000));
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
  const double A_INab = (q->PNab * q->ffrt * (S[nai] * exp(vfrt) - q->nao)) / q->B_INab;
  const double U_INab = q->B_INab * (v - q->v0_INab);
  const double INab = (-1.00000e-07 <= U_INab && U_INab <= 1.00000e-07 ? A_INab * (1.00000 - 0.500000 * U_INab)
                                                                       : (A_INab * U_INab) / (exp(U_INab) - 1.00000));
  const double JdiffNa = (S[nass] - S[nai]) / 2.00000;
  const double A_2 = (0.750000 * q->ffrt * (S[nass] * exp(vfrt) - q->nao)) / q->B_2;
  const double U_2 = q->B_2 * (v - q->v0);
  const double PhiCaNa = (-1.00000e-07 <= U_2 && U_2 <= 1.00000e-07 ? A_2 * (1.00000 - 0.500000 * U_2)
                                                                    : (A_2 * U_2) / (exp(U_2) - 1.00000));
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
  const double A_ICab = (q->PCab * 4.00000 * q->ffrt * (S[cai] * exp(2.00000 * vfrt) - 0.341000 * q->cao)) / q->B_ICab;
  const double U_ICab = q->B_ICab * (v - q->v0_ICab);
  const double ICab = (-1.00000e-07 <= U_ICab && U_ICab <= 1.00000e-07 ? A_ICab * (1.00000 - 0.500000 * U_ICab)
                                                                       : (A_ICab * U_ICab) / (exp(U_ICab) - 1.00000));
  const double Jdiff = (S[cass] - S[cai]) / 0.200000;
  const double fJrelp = 1.00000 / (1.00000 + q->KmCaMK / CaMKa);
  const double Jrel = q->Jrel_scaling_factor * ((1.00000 - fJrelp) * S[Jrelnp] + fJrelp * S[Jrelp]);
  const double Bcass = 1.00000 / (1.00000 + (q->BSRmax * q->KmBSR) / pow(q->KmBSR + S[cass], 2.00000) +
                                  (q->BSLmax * q->KmBSL) / pow(q->KmBSL + S[cass], 2.00000));
  const double Jupnp = (q->upScale * 0.00437500 * S[cai]) / (S[cai] + 0.000920000);
  const double Jupp = (q->upScale * 2.75000 * 0.00437500 * S[cai]) / ((S[cai] + 0.000920000) - 0.000170000);
  const double fJupp = 1.00000 / (1.00000 + q->KmCaMK / CaMKa);
  const double Jleak = (0.00393750 * S[cansr]) / 15.0000;
  const double Jup = q->Jup_b * (((1.00000 - fJupp) * Jupnp + fJupp * Jupp) - Jleak);
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
    R_[xs1] = (g->xs1ss - S[xs1]) / g->txs1;
    R_[xk1] = (g->xk1ss - S[xk1]) / g->txk1;
    R_[CaMKt] = q->aCaMK * CaMKb * (CaMKb + S[CaMKt]) - q->bCaMK * S[CaMKt];
    R_[j] = (g->jss - S[j]) / g->tj;
    R_[ap] = (g->assp - S[ap]) / g->ta;
    R_[fcaf] = (g->fcass - S[fcaf]) / g->tfcaf;
    R_[fcas] = (g->fcass - S[fcas]) / g->tfcas;
    R_[ffp] = (g->fss - S[ffp]) / g->tffp;
    R_[xs2] = (g->xs2ss - S[xs2]) / g->txs2;
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
    cur->INa = INa; cur->INaL = INaL; cur->Ito = Ito; cur->ICaL = ICaL; cur->IKr = IKr; cur->IKs = IKs;
    cur->IK1 = IK1; cur->dVdt = R_ ? R_[V] : 0.0;
  }
}

void cepo_cipa_rates(const cepo_cell *c, double t, const double *y, double *dydt, cepo_currents *cur) {
  double r[CIPA_NS];
  double yy[CIPA_NS];
  cipa_gates g;
  memcpy(yy, y, sizeof(yy));
  yy[Dst] = ((const cipa_p *)c->p)->D;
  cipa_compute(c, t, yy, dydt ? dydt : r, &g, cur);
}

#define RL(y, inf, tau) ((inf) - ((inf) - (y)) * exp(-dt / (tau)))

/* One backward-Euler step of the Markov IKr chain (the rates frozen at the
 * step's V): (I - dt Q) x = g with g = dt Q S the forward-Euler increments,
 * S += x. The chain's graph is sparse, so the 9x9 system is eliminated in a
 * fixed order: Cb, the bound pair {Ob, IOb} (2x2, in terms of O and IO),
 * IC1, C1, C2, then the dense 3x3 {IC2, O, IO}. I - dt Q is an M-matrix
 * (columns of Q sum to zero), so no pivoting is needed, and the step keeps
 * the chain's total occupancy exactly. k[] = {k11, k21, k51, k61, k3, k4,
 * k52, k62, k1, k2, k31, k41, k53, k63, bind, Ku, unb, trap, Kt}. */
static void markov_backward_euler(double h, const double *k, const double *g, double *x) {
  const double k11 = k[0], k21 = k[1], k51 = k[2], k61 = k[3], k3 = k[4], k4 = k[5], k52 = k[6], k62 = k[7];
  const double k1 = k[8], k2 = k[9], k31 = k[10], k41 = k[11], k53 = k[12], k63 = k[13], bind = k[14];
  const double Ku = k[15], unb = k[16], trap = k[17], Kt = k[18];
  /* g and x in state order IC1, IC2, C1, C2, O, IO, IObound, Obound, Cbound */
  const double dIC1 = 1.0 + h * (k11 + k61), dIC2 = 1.0 + h * ((k21 + k3) + k62), dC1 = 1.0 + h * (k51 + k1);
  const double dC2 = 1.0 + h * ((k2 + k52) + k31), dO = 1.0 + h * ((k41 + k53) + bind);
  const double dIO = 1.0 + h * ((k4 + k63) + bind), dIOb = 1.0 + h * (unb + Kt), dOb = 1.0 + h * (Ku + Kt);
  const double dCb = 1.0 + h * (2.0 * trap);
  /* Cb, then the bound pair as affine functions of dO, dIO */
  const double ht = h * trap, hK = h * Kt, hb = h * bind;
  const double c = ht * hK / dCb, e = ht * g[8] / dCb;
  const double a11 = dOb - c, a22 = dIOb - c, det = a11 * a22 - c * c;
  const double rOb = g[7] + e, rIOb = g[6] + e;
  const double ob0 = (a22 * rOb + c * rIOb) / det, obO = a22 * hb / det, obIO = c * hb / det;
  const double iob0 = (c * rOb + a11 * rIOb) / det, iobO = c * hb / det, iobIO = a11 * hb / det;
  const double aOO = dO - h * Ku * obO, aOIO = -(h * k63 + h * Ku * obIO), aOC2 = -h * k31;
  const double rO = g[4] + h * Ku * ob0;
  const double aIOIO = dIO - h * unb * iobIO, aIOO = -(h * k53 + h * unb * iobO), aIOIC2 = -h * k3;
  const double rIO = g[5] + h * unb * iob0;
  /* IC1 and C1 as affine functions of IC2, C2 */
  const double i0 = g[0] / dIC1, iI2 = h * k21 / dIC1, iC1 = h * k51 / dIC1;
  const double e11 = dC1 - h * k61 * iC1;
  const double c0 = (g[2] + h * k61 * i0) / e11, cI2 = h * k61 * iI2 / e11, cC2 = h * k2 / e11;
  const double bII = dIC2 - h * k11 * (iI2 + iC1 * cI2), bIC = -(h * k52 + h * k11 * iC1 * cC2);
  const double bIIO = -h * k4, rI = g[1] + h * k11 * (i0 + iC1 * c0);
  const double bCC = dC2 - h * k1 * cC2, bCI = -(h * k62 + h * k1 * cI2), bCO = -h * k41;
  const double rC = g[3] + h * k1 * c0;
  /* C2 out, then the 3x3 {IC2, O, IO} */
  const double m11 = bII - bIC * bCI / bCC, m12 = -bIC * bCO / bCC, m13 = bIIO, s1 = rI - bIC * rC / bCC;
  const double m21 = -aOC2 * bCI / bCC, m22 = aOO - aOC2 * bCO / bCC, m23 = aOIO, s2 = rO - aOC2 * rC / bCC;
  const double m31 = aIOIC2, m32 = aIOO, m33 = aIOIO, s3 = rIO;
  const double l21 = m21 / m11, l31 = m31 / m11;
  const double n22 = m22 - l21 * m12, n23 = m23 - l21 * m13, t2 = s2 - l21 * s1;
  const double n32 = m32 - l31 * m12, n33 = m33 - l31 * m13, t3 = s3 - l31 * s1;
  const double l32 = n32 / n22;
  const double xIO = (t3 - l32 * t2) / (n33 - l32 * n23);
  const double xO = (t2 - n23 * xIO) / n22;
  const double xIC2 = ((s1 - m12 * xO) - m13 * xIO) / m11;
  const double xC2 = ((rC - bCI * xIC2) - bCO * xO) / bCC;
  const double xC1 = (c0 + cI2 * xIC2) + cC2 * xC2;
  const double xOb = (ob0 + obO * xO) + obIO * xIO, xIOb = (iob0 + iobO * xO) + iobIO * xIO;
  x[0] = (i0 + iI2 * xIC2) + iC1 * xC1;
  x[1] = xIC2; x[2] = xC1; x[3] = xC2; x[4] = xO; x[5] = xIO; x[6] = xIOb; x[7] = xOb;
  x[8] = (g[8] + hK * (xIOb + xOb)) / dCb;
}

/* Fixed-step scheme: Rush-Larsen gates, forward Euler for the Markov IKr
 * states, V, ions and CaMKII (the ORd scheme, Ohara_Rudy_2011.cpp:1036-1094). */
void cepo_cipa_step(const cepo_cell *c, double t, double dt, double *S, cepo_currents *cur) {
  const cipa_p *q = (const cipa_p *)c->p;
  double R_[CIPA_NS];
  cipa_gates g;
  S[Dst] = q->D;
  cipa_compute(c, t, S, R_, &g, cur);
  S[m] = RL(S[m], g.mss, g.tm);
  S[hf] = RL(S[hf], g.hss, g.thf);
  S[hs] = RL(S[hs], g.hss, g.ths);
  S[j] = RL(S[j], g.jss, g.tj);
  S[hsp] = RL(S[hsp], g.hssp, g.thsp);
  S[jp] = RL(S[jp], g.jss, g.tjp);
  S[mL] = RL(S[mL], g.mLss, g.tmL);
  S[hL] = RL(S[hL], g.hLss, q->thL);
  S[hLp] = RL(S[hLp], g.hLssp, q->thLp);
  S[a] = RL(S[a], g.ass, g.ta);
  S[iF] = RL(S[iF], g.iss, g.tiF);
  S[iS] = RL(S[iS], g.iss, g.tiS);
  S[ap] = RL(S[ap], g.assp, g.ta);
  S[iFp] = RL(S[iFp], g.iss, g.tiFp);
  S[iSp] = RL(S[iSp], g.iss, g.tiSp);
  S[d] = RL(S[d], g.dss, g.td);
  S[ff] = RL(S[ff], g.fss, g.tff);
  S[fs] = RL(S[fs], g.fss, g.tfs);
  S[fcaf] = RL(S[fcaf], g.fcass, g.tfcaf);
  S[fcas] = RL(S[fcas], g.fcass, g.tfcas);
  S[jca] = RL(S[jca], g.fcass, q->tjca);
  S[ffp] = RL(S[ffp], g.fss, g.tffp);
  S[fcafp] = RL(S[fcafp], g.fcass, g.tfcafp);
  S[nca] = g.anca * q->k2n / g.km2n - (g.anca * q->k2n / g.km2n - S[nca]) * exp(-g.km2n * dt);
  S[xs1] = RL(S[xs1], g.xs1ss, g.txs1);
  S[xs2] = RL(S[xs2], g.xs2ss, g.txs2);
  S[xk1] = RL(S[xk1], g.xk1ss, g.txk1);
  S[Jrelnp] = RL(S[Jrelnp], g.Jrel_inf, g.tau_rel);
  S[Jrelp] = RL(S[Jrelp], g.Jrel_infp, g.tau_relp);
  /* Markov IKr states: forward Euler, as the reference scheme treats every
   * non-gate state. The chain is linear in its states for the step's V; when
   * its largest outflow rate lam makes the Euler step unsafe (dt*lam > 1.8:
   * fast drug binding, the IC2 -> IC1 rate below ~-95 mV, IC1 -> C1 above
   * ~43 mV) the step is one backward-Euler step of the chain instead
   * (stable for any rate, total occupancy kept). */
  if (dt * g.lam_max <= 1.8) {
    S[IC1] = S[IC1] + R_[IC1] * dt;
    S[IC2] = S[IC2] + R_[IC2] * dt;
    S[C1] = S[C1] + R_[C1] * dt;
    S[C2] = S[C2] + R_[C2] * dt;
    S[O] = S[O] + R_[O] * dt;
    S[IO] = S[IO] + R_[IO] * dt;
    S[IObound] = S[IObound] + R_[IObound] * dt;
    S[Obound] = S[Obound] + R_[Obound] * dt;
    S[Cbound] = S[Cbound] + R_[Cbound] * dt;
  } else {
    const double kk[19] = {g.e11 * Q10(q->q11), g.e21 * Q10(q->q21), g.e51 * Q10(q->q51), g.e61 * Q10(q->q61),
                           g.e3 * Q10(q->q3),   g.e4 * Q10(q->q4),   g.e52 * Q10(q->q52), g.e62 * Q10(q->q62),
                           g.e1 * Q10(q->q1),   g.e2 * Q10(q->q2),   g.e31 * Q10(q->q31), g.e41 * Q10(q->q41),
                           g.e53 * Q10(q->q53), g.e63 * Q10(q->q63), g.bind, q->Ku, g.unb, g.trap, q->Kt};
    const double gg[9] = {R_[IC1] * dt, R_[IC2] * dt, R_[C1] * dt, R_[C2] * dt, R_[O] * dt, R_[IO] * dt,
                          R_[IObound] * dt, R_[Obound] * dt, R_[Cbound] * dt};
    double x[9];
    markov_backward_euler(dt, kk, gg, x);
    S[IC1] += x[0]; S[IC2] += x[1]; S[C1] += x[2]; S[C2] += x[3]; S[O] += x[4];
    S[IO] += x[5]; S[IObound] += x[6]; S[Obound] += x[7]; S[Cbound] += x[8];
  }
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
int cepo_cipa_scale(cepo_cell *c, int g, double f) {
  cipa_p *q = (cipa_p *)c->p;
  double *x = g == 0 ? &q->GNa : g == 1 ? &q->GNaL : g == 2 ? &q->Gto : g == 3 ? &q->PCa : g == 4 ? &q->GKr
            : g == 5 ? &q->GKs : g == 6 ? &q->GK1 : g == 11 ? &q->GKb : g == 12 ? &q->Gncx : g == 13 ? &q->Pnak : 0;
  if (!x) return -1;
  *x *= f;
  return 0;
}
