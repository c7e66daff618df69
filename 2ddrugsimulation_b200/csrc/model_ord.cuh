// O'Hara-Rudy 2011 and CiPA-ORd v1 2017 ventricular models, register-
// resident state, templated on the precision policy (cep_device.cuh).
//
// Equations and update scheme: DrugSimulation/cellmodels/Ohara_Rudy_2011.cpp
// computeRates (:742-989) and the Rush-Larsen / forward-Euler branch of
// solveAnalytical (:1036-1094). Model constants that do not depend on the
// instance are compile-time constants here; the per-instance ones (celltype
// scalings, Dutta scalings, Hill-scaled conductances, pacing) come from the
// parameter block built by ord_init_kernel.
#pragma once
#include "cep_device.cuh"

namespace cep {
namespace ord {

constexpr int kNumStates = 41;

// STATES order of the reference (enums/enum_Ohara_Rudy_2011.hpp), which is
// also the order of the C-ABI state arrays.
enum : int {
  V = 0, CaMKt, cass, nai, nass, ki, kss, cansr, cajsr, cai, m, hf, hs, j, hsp, jp, mL, hL, hLp, a,
  iF, iS, ap, iFp, iSp, d, ff, fs, fcaf, fcas, jca, ffp, fcafp, nca, xrf, xrs, xs1, xs2, xk1,
  Jrelnp, Jrelp
};

// CiPA-ORd v1 2017 STATES order (enums/enum_ohara_rudy_cipa_v1_2017.hpp):
// the ORd states without xrf/xrs, the nine Markov IKr states and the drug
// concentration D.
namespace cipa {
constexpr int kNumStates = 49;
enum : int {
  V = 0, CaMKt, cass, nai, nass, ki, kss, cansr, cajsr, cai, m, hf, hs, j, hsp, jp, mL, hL, hLp, a, iF,
  iS, ap, iFp, iSp, d, ff, fs, fcaf, fcas, jca, ffp, fcafp, nca, IC1, IC2, C1, C2, O, IO, IObound, Obound,
  Cbound, D, xs1, xs2, xk1, Jrelnp, Jrelp
};
// Q10 factors exp(((37 - 20) * log(q)) / 10) of the hERG transitions
// (ohara_rudy_cipa_v1_2017.cpp:2157-2165), evaluated once in FP64.
constexpr double Q1 = 14.611493102188247, Q2 = 11.608567327201762, Q3 = 15.227075177403329;
constexpr double Q4 = 9.540792127868109, Q11 = 15.122885354397773, Q21 = 11.265446673074576;
constexpr double Q31 = 11.561952122102017, Q41 = 1.9006143161790194, Q51 = 15.425846568000235;
constexpr double Q52 = 13.700335619455835, Q53 = 4.4672619154839515, Q61 = 18.522034347349482;
constexpr double Q62 = 15.425846568000235, Q63 = 19.171323250640047;
// A and B of the transition rates A*exp(B*V)*Q (active ___initConsts block)
constexpr double A1 = 0.0264, B1 = 4.631E-05, A2 = 4.986E-06, B2 = -0.004226, A3 = 0.001214, B3 = 0.008516;
constexpr double A4 = 1.854E-05, B4 = -0.04641, A11 = 0.0007868, B11 = 1.535E-08, A21 = 5.455E-06;
constexpr double B21 = -0.1688, A31 = 0.005509, B31 = 7.771E-09, A41 = 0.001416, B41 = -0.02877;
constexpr double A51 = 0.4492, B51 = 0.008595, A52 = 0.3181, B52 = 3.613E-08, A53 = 0.149, B53 = 0.004668;
constexpr double A61 = 0.01241, B61 = 0.1725, A62 = 0.3226, B62 = -0.0006575, A63 = 0.008978, B63 = -0.02215;
}  // namespace cipa

// Per-instance parameter block (one SoA row per entry).
enum : int {
  P_GNa = 0, P_GNaL, P_Gto, P_PCa, P_PCap, P_PCaNa, P_PCaK, P_PCaNap, P_PCaKp, P_GKr, P_GKs, P_GK1,
  P_GKb, P_Gncx, P_Pnak, P_cmdnmax, P_upScale, P_Aff, P_Afs, P_tjca, P_H, P_celltype, P_fcafp_dt,
  P_amp, P_BCL, P_stim_start, P_duration,
  P_bind, P_Ku, P_Kt, P_Vhalf,  // CiPA dynamic hERG drug binding
  kNumParams
};

// Instance-independent constants of ___initConsts (Ohara_Rudy_2011.cpp:494-678).
namespace k {
constexpr double nao = 140, cao = 1.8, ko = 5.4, R = 8314, T = 310, F = 96485, zna = 1, zca = 2, zk = 1;
constexpr double L = 0.01, rad = 0.0011;
constexpr double KmCaMK = 0.15, aCaMK = 0.05, bCaMK = 0.00068, CaMKo = 0.05, KmCaM = 0.0015;
constexpr double kmcmdn = 0.00238, trpnmax = 0.07, kmtrpn = 0.0005, BSRmax = 0.047, KmBSR = 0.00087;
constexpr double BSLmax = 1.124, KmBSL = 0.0087, csqnmax = 10, kmcsqn = 0.8, cm = 1, PKNa = 0.01833;
constexpr double mssV1 = 39.57, mssV2 = 9.871, mtV1 = 11.64, mtV2 = 34.77, mtD1 = 6.765, mtD2 = 8.552;
constexpr double mtV3 = 77.42, mtV4 = 5.955, hssV1 = 82.9, hssV2 = 6.086, Ahf = 0.99, Ahs = 1.0 - Ahf;
constexpr double thL = 200, thLp = 3.0 * thL, Kmn = 0.002, k2n = 1000;
constexpr double kna1 = 15, kna2 = 5, kna3 = 88.12, kasymm = 12.5, wna = 6e4, wca = 6e4, wnaca = 5e3;
constexpr double kcaon = 1.5e6, kcaoff = 5e3, qna = 0.5224, qca = 0.167, KmCaAct = 150e-6;
constexpr double k1p = 949.5, k1m = 182.4, k2p = 687.2, k2m = 39.4, k3p = 1899, k3m = 79300, k4p = 639;
constexpr double k4m = 40, Knai0 = 9.073, Knao0 = 27.78, delta = -0.155, Kki = 0.5, Kko = 0.3582;
constexpr double MgADP = 0.05, MgATP = 9.8, Kmgatp = 1.698e-7, eP = 4.2, Khp = 1.698e-7, Knap = 224;
constexpr double Kxkur = 292, PNab = 3.75e-10, PCab = 2.5e-8, GpCa = 0.0005, KmCap = 0.0005, bt = 4.75;
constexpr double a_rel = 0.5 * bt, btp = 1.25 * bt, a_relp = 0.5 * btp;
constexpr double vcell = 1000.00 * 3.14000 * rad * rad * L;
constexpr double Ageo = 2.0 * 3.14 * rad * rad + 2.0 * 3.14 * rad * L;
constexpr double Acap = 2.0 * Ageo, vmyo = 0.68 * vcell, vnsr = 0.0552 * vcell;
constexpr double vjsr = 0.0048 * vcell, vss = 0.02 * vcell;
constexpr double h10 = kasymm + 1.0 + (nao / kna1) * (1.0 + nao / kna2);
constexpr double h11 = (nao * nao) / (h10 * kna1 * kna2);
constexpr double h12 = 1.0 / h10;
constexpr double k1x = h12 * cao * kcaon, k2x = kcaoff, k5x = kcaoff;
constexpr double b1 = k1m * MgADP, a2 = k2p;
constexpr double a4 = ((k4p * MgATP) / Kmgatp) / (1.0 + MgATP / Kmgatp);
constexpr double RTF = (R * T) / F;           // mV
constexpr double FRT = F / (R * T);           // 1/mV
constexpr double FFRT = F * F / (R * T);
// ionic flux scalings of the RATES expressions
constexpr double cAF_myo = cm * Acap / (F * vmyo), cAF_ss = cm * Acap / (F * vss);
constexpr double sqrt_ko54 = 1.0;  // pow(ko/5.4, 1/2) with ko = 5.4
constexpr double sqrt_ko = 2.32379000772445;  // pow(5.4, 1/2)
constexpr double xk1_off = 2.55380 * ko + 144.590, xk1_den = 1.56920 * ko + 3.81150;
constexpr double a3c = k3p * (ko / Kko) * (ko / Kko), ko_Kko_sq = (1.0 + ko / Kko) * (1.0 + ko / Kko);
// Mixed-policy shortcuts (one SFU op each): gates whose steady states share
// a slope differ by a constant factor of the exponential,
// e^((V+89.1)/6.086) = e^((V+82.9)/6.086) e^(6.2/6.086) (hssp vs hss),
// e^((V+93.81)/7.488) = e^((V+87.61)/7.488) e^(6.2/7.488) (hLssp vs hLss),
// e^(-(V-24.34)/14.82) = e^(-(V-14.34)/14.82) e^(10/14.82) (assp vs ass);
// and log(c_o/c_i) = log(c_o) - log(c_i) for ENa and EK.
constexpr double hssp_shift = 2.769679238039406, hLssp_shift = 2.288717124596483, assp_shift = 1.9635691902911017;
constexpr double log_nao = 4.941642422609304, log_ko = 1.6863989535702288;
// log(ko + PKNa nao) for EKs, log(3.8e-5) for the IKs calcium factor
constexpr double log_ks_o = 2.0752075911477745, log_ks_ca = -10.177924398237888;
}  // namespace k

template <class G>
struct Y {
  // every state is stored in FP64; the mixed path computes from FP32 copies
  double V, CaMKt, cass, nai, nass, ki, kss, cansr, cajsr, cai;
  double m, hf, hs, j, hsp, jp, mL, hL, hLp, a, iF, iS, ap, iFp, iSp, d, ff, fs, fcaf, fcas, jca, ffp,
      fcafp, nca, xrf, xrs, xs1, xs2, xk1, Jrelnp, Jrelp;
  double IC1, IC2, C1, C2, O, IO, IObound, Obound, Cbound;  // CiPA Markov IKr
};

template <class G>
struct Par {
  G GNa, GNaL, Gto, PCa, PCap, PCaNa, PCaK, PCaNap, PCaKp, GKr, GKs, GK1, GKb, Gncx, Pnak;
  G cmdnmax, upScale, Aff, Afs, tjca, b3c;
  G fcafp_dt;  // 0: use dt
  int celltype;
  double amp, BCL, stim_start, duration;
  G bind, Ku, Kt, Vhalf;  // CiPA: Kmax*Ku*D^n/(D^n + halfmax), unbinding, trapping
};

template <class G>
struct Cur {
  G INa, INaL, Ito, ICaL, IKr, IKs, IK1, dVdt;
};

// Loads/stores between the SoA arrays [kNumStates][ld] and registers.
template <class G>
__device__ __forceinline__ void load(Y<G> &y, const double *__restrict__ s, int64_t ld, int64_t i) {
  y.V = s[V * ld + i]; y.CaMKt = s[CaMKt * ld + i]; y.cass = s[cass * ld + i];
  y.nai = s[nai * ld + i]; y.nass = s[nass * ld + i]; y.ki = s[ki * ld + i];
  y.kss = s[kss * ld + i]; y.cansr = s[cansr * ld + i]; y.cajsr = s[cajsr * ld + i];
  y.cai = s[cai * ld + i];
#define CEP_LD(n) y.n = s[n * ld + i];
  CEP_LD(m) CEP_LD(hf) CEP_LD(hs) CEP_LD(j) CEP_LD(hsp) CEP_LD(jp) CEP_LD(mL) CEP_LD(hL) CEP_LD(hLp)
  CEP_LD(a) CEP_LD(iF) CEP_LD(iS) CEP_LD(ap) CEP_LD(iFp) CEP_LD(iSp) CEP_LD(d) CEP_LD(ff) CEP_LD(fs)
  CEP_LD(fcaf) CEP_LD(fcas) CEP_LD(jca) CEP_LD(ffp) CEP_LD(fcafp) CEP_LD(nca) CEP_LD(xrf) CEP_LD(xrs)
  CEP_LD(xs1) CEP_LD(xs2) CEP_LD(xk1) CEP_LD(Jrelnp) CEP_LD(Jrelp)
#undef CEP_LD
}

template <class G>
__device__ __forceinline__ void store(const Y<G> &y, double *__restrict__ s, int64_t ld, int64_t i) {
  s[V * ld + i] = y.V; s[CaMKt * ld + i] = y.CaMKt; s[cass * ld + i] = y.cass;
  s[nai * ld + i] = y.nai; s[nass * ld + i] = y.nass; s[ki * ld + i] = y.ki;
  s[kss * ld + i] = y.kss; s[cansr * ld + i] = y.cansr; s[cajsr * ld + i] = y.cajsr;
  s[cai * ld + i] = y.cai;
#define CEP_ST(n) s[n * ld + i] = y.n;
  CEP_ST(m) CEP_ST(hf) CEP_ST(hs) CEP_ST(j) CEP_ST(hsp) CEP_ST(jp) CEP_ST(mL) CEP_ST(hL) CEP_ST(hLp)
  CEP_ST(a) CEP_ST(iF) CEP_ST(iS) CEP_ST(ap) CEP_ST(iFp) CEP_ST(iSp) CEP_ST(d) CEP_ST(ff) CEP_ST(fs)
  CEP_ST(fcaf) CEP_ST(fcas) CEP_ST(jca) CEP_ST(ffp) CEP_ST(fcafp) CEP_ST(nca) CEP_ST(xrf) CEP_ST(xrs)
  CEP_ST(xs1) CEP_ST(xs2) CEP_ST(xk1) CEP_ST(Jrelnp) CEP_ST(Jrelp)
#undef CEP_ST
}

template <class G>
__device__ __forceinline__ void load_par(Par<G> &q, const double *__restrict__ p, int64_t ld, int64_t i) {
  q.GNa = (G)p[P_GNa * ld + i]; q.GNaL = (G)p[P_GNaL * ld + i]; q.Gto = (G)p[P_Gto * ld + i];
  q.PCa = (G)p[P_PCa * ld + i]; q.PCap = (G)p[P_PCap * ld + i]; q.PCaNa = (G)p[P_PCaNa * ld + i];
  q.PCaK = (G)p[P_PCaK * ld + i]; q.PCaNap = (G)p[P_PCaNap * ld + i];
  q.PCaKp = (G)p[P_PCaKp * ld + i]; q.GKr = (G)p[P_GKr * ld + i]; q.GKs = (G)p[P_GKs * ld + i];
  q.GK1 = (G)p[P_GK1 * ld + i]; q.GKb = (G)p[P_GKb * ld + i]; q.Gncx = (G)p[P_Gncx * ld + i];
  q.Pnak = (G)p[P_Pnak * ld + i]; q.cmdnmax = (G)p[P_cmdnmax * ld + i];
  q.upScale = (G)p[P_upScale * ld + i]; q.Aff = (G)p[P_Aff * ld + i]; q.Afs = (G)p[P_Afs * ld + i];
  q.tjca = (G)p[P_tjca * ld + i];
  // b3 = k3m * P * H / (1 + MgATP/Kmgatp): fold the instance's H (the Dutta
  // quirk scales H) into one factor.
  q.b3c = (G)((k::k3m * 1.0) * p[P_H * ld + i] / (1.0 + k::MgATP / k::Kmgatp));
  q.fcafp_dt = (G)p[P_fcafp_dt * ld + i];
  q.celltype = (int)p[P_celltype * ld + i];
  q.amp = p[P_amp * ld + i]; q.BCL = p[P_BCL * ld + i];
  q.stim_start = p[P_stim_start * ld + i]; q.duration = p[P_duration * ld + i];
  q.bind = (G)p[P_bind * ld + i]; q.Ku = (G)p[P_Ku * ld + i]; q.Kt = (G)p[P_Kt * ld + i];
  q.Vhalf = (G)p[P_Vhalf * ld + i];
}

// CiPA state layout <-> registers
template <class G>
__device__ __forceinline__ void load_cipa(Y<G> &y, const double *__restrict__ s, int64_t ld, int64_t i) {
#define CEP_LD(n) y.n = s[cipa::n * ld + i];
  CEP_LD(V) CEP_LD(CaMKt) CEP_LD(cass) CEP_LD(nai) CEP_LD(nass) CEP_LD(ki) CEP_LD(kss) CEP_LD(cansr)
  CEP_LD(cajsr) CEP_LD(cai) CEP_LD(m) CEP_LD(hf) CEP_LD(hs) CEP_LD(j) CEP_LD(hsp) CEP_LD(jp) CEP_LD(mL)
  CEP_LD(hL) CEP_LD(hLp) CEP_LD(a) CEP_LD(iF) CEP_LD(iS) CEP_LD(ap) CEP_LD(iFp) CEP_LD(iSp) CEP_LD(d)
  CEP_LD(ff) CEP_LD(fs) CEP_LD(fcaf) CEP_LD(fcas) CEP_LD(jca) CEP_LD(ffp) CEP_LD(fcafp) CEP_LD(nca)
  CEP_LD(IC1) CEP_LD(IC2) CEP_LD(C1) CEP_LD(C2) CEP_LD(O) CEP_LD(IO) CEP_LD(IObound) CEP_LD(Obound)
  CEP_LD(Cbound) CEP_LD(xs1) CEP_LD(xs2) CEP_LD(xk1) CEP_LD(Jrelnp) CEP_LD(Jrelp)
#undef CEP_LD
  y.xrf = 0.0; y.xrs = 0.0;
}

template <class G>
__device__ __forceinline__ void store_cipa(const Y<G> &y, double *__restrict__ s, int64_t ld, int64_t i) {
#define CEP_ST(n) s[cipa::n * ld + i] = y.n;
  CEP_ST(V) CEP_ST(CaMKt) CEP_ST(cass) CEP_ST(nai) CEP_ST(nass) CEP_ST(ki) CEP_ST(kss) CEP_ST(cansr)
  CEP_ST(cajsr) CEP_ST(cai) CEP_ST(m) CEP_ST(hf) CEP_ST(hs) CEP_ST(j) CEP_ST(hsp) CEP_ST(jp) CEP_ST(mL)
  CEP_ST(hL) CEP_ST(hLp) CEP_ST(a) CEP_ST(iF) CEP_ST(iS) CEP_ST(ap) CEP_ST(iFp) CEP_ST(iSp) CEP_ST(d)
  CEP_ST(ff) CEP_ST(fs) CEP_ST(fcaf) CEP_ST(fcas) CEP_ST(jca) CEP_ST(ffp) CEP_ST(fcafp) CEP_ST(nca)
  CEP_ST(IC1) CEP_ST(IC2) CEP_ST(C1) CEP_ST(C2) CEP_ST(O) CEP_ST(IO) CEP_ST(IObound) CEP_ST(Obound)
  CEP_ST(Cbound) CEP_ST(xs1) CEP_ST(xs2) CEP_ST(xk1) CEP_ST(Jrelnp) CEP_ST(Jrelp)
#undef CEP_ST
}

// Periodic single-cell stimulus of computeRates (Ohara_Rudy_2011.cpp:747);
// stim_mode >= 0 selects the tissue form (isS1, :745).
__device__ __forceinline__ bool stim_on(double t, double start, double bcl, double dur) {
  return t >= start && (t - start) - floor((t - start) / bcl) * bcl <= dur;
}

// ---------------------------------------------------------------------------
// One cell step, organised in four roles plus a combine stage.
//
// Every role reads the FP64 state (V, ions, CaMKII) and owns a disjoint set
// of gates, which it advances with Rush-Larsen; it returns its contribution
// to the membrane and flux sums in a Part. combine() adds the four Parts in
// a fixed order and advances the FP64 states with forward Euler. The same
// role functions serve the one-thread-per-cell kernel (step(): the roles run
// back to back) and the warp-specialised kernel (one warp per role for 32
// cells, Parts exchanged through shared memory); both add the Parts in the
// same order.
//   role 0 (Na): m hf hs j hsp jp mL hL hLp; INa, INaL, INab, INaK
//   role 1 (K) : a iF iS ap iFp iSp xs1 xs2 (ORd: xrf xrs); Ito, IKs, IKb,
//                IKr (ORd), Istim
//   xk1 and IK1 go to role 0 in FP64 and to role 1 in the mixed path
//   (kIK1InNa)
//   role 2 (Ca): d ff fs fcaf fcas jca ffp fcafp nca Jrelnp Jrelp; ICaL, ICaNa,
//                ICaK, ICab, IpCa, Jrel
//   role 3 (X) : INaCa_i, INaCa_ss, Jup; CiPA: the Markov IKr chain and IKr
// ---------------------------------------------------------------------------

// Contributions to the sums the forward-Euler update needs
// (Ohara_Rudy_2011.cpp:962-988 RATES of V and the ions).
enum : int {
  S_iV = 0,   // sum of the membrane currents, Istim included (RATES[V] = -iV)
  S_iNa,      // INa + INaL + 3 INaCa_i + 3 INaK + INab       (nai)
  S_iNass,    // ICaNa + 3 INaCa_ss                            (nass)
  S_iK,       // Ito + IKr + IKs + IK1 + IKb + Istim - 2 INaK  (ki)
  S_iKss,     // ICaK                                           (kss)
  S_iCass,    // ICaL - 2 INaCa_ss                             (cass)
  S_iCai,     // IpCa + ICab - 2 INaCa_i                       (cai)
  S_Jrel, S_Jup,
  S_INa, S_INaL, S_ICaL, S_Ito, S_IKr, S_IKs, S_IK1,  // reported currents
  kNumSums
};

template <class G>
struct Part {
  G f[kNumSums];
};

// Where IK1 and its gate xk1 are evaluated: the Na group in FP64, where the
// K group has the longest dependency chain of the four (measured with clock
// stamps per group: 8,400 cycles per step against 6,000-7,000); the K group
// in the mixed path, whose pairs form carries Na + Ca in one warp and K + the
// rest in the other and is balanced that way.
template <class P>
inline constexpr bool kIK1InNa = !P::kMixed;

// Fields each role writes, in the order of its packed shared-memory slot
// (at most 8; -1 = unused).
template <bool kIK1Na>
__host__ __device__ constexpr int role_field(int role, int k) {
  constexpr int a[4][8] = {{S_iV, S_iNa, S_iK, S_INa, S_INaL, S_IK1, -1, -1},
                           {S_iV, S_iK, S_Ito, S_IKr, S_IKs, -1, -1, -1},
                           {S_iV, S_iNass, S_iKss, S_iCass, S_iCai, S_Jrel, S_ICaL, -1},
                           {S_iV, S_iNa, S_iNass, S_iCass, S_iCai, S_Jup, S_IKr, S_iK}};
  constexpr int b[4][8] = {{S_iV, S_iNa, S_iK, S_INa, S_INaL, -1, -1, -1},
                           {S_iV, S_iK, S_Ito, S_IKr, S_IKs, S_IK1, -1, -1},
                           {S_iV, S_iNass, S_iKss, S_iCass, S_iCai, S_Jrel, S_ICaL, -1},
                           {S_iV, S_iNa, S_iNass, S_iCass, S_iCai, S_Jup, S_IKr, S_iK}};
  return kIK1Na ? a[role][k] : b[role][k];
}

// Values every role needs at the start of a step.
template <class G>
struct Ctx {
  G v;       // membrane potential in the working precision
  G fCaMKp;  // fraction of phosphorylated channels 1/(1 + KmCaMK/CaMKa)
  bool stim;
};

template <class P>
__device__ __forceinline__ Ctx<typename P::G> context(const Y<typename P::G> &y, const Par<typename P::G> &q,
                                                      double t, int stim_mode) {
  using G = typename P::G;
  Ctx<G> c;
  c.v = (G)y.V;
  // mixed: a/(1 + K/c) as a c/(c + K), one division for two
  const G cass = (G)y.cass;
  const G CaMKb = P::kFast ? P::dv((G)k::CaMKo * ((G)1 - (G)y.CaMKt) * cass, cass + (G)k::KmCaM)
                            : P::dv(((G)k::CaMKo * ((G)1 - (G)y.CaMKt)), ((G)1 + P::dv((G)k::KmCaM, cass)));
  const G CaMKa = CaMKb + (G)y.CaMKt;
  c.fCaMKp = P::kFast ? P::dv(CaMKa, CaMKa + (G)k::KmCaMK) : P::rc(((G)1 + P::dv((G)k::KmCaMK, CaMKa)));
  c.stim = stim_mode < 0 ? stim_on(t, q.stim_start, q.BCL, q.duration) : (stim_mode != 0);
  return c;
}

// GHK factor for a flux of valence z at V: the reference's ORd form
// vffrt/(e^{z vfrt} - 1) scaled by z (ORd, FP64), the CiPA-v1 form A*U/(e^U-1)
// with the |U| <= 1e-7 guard (CiPA, FP64), or the stable x/(e^x - 1) form
// (mixed). Returns (flux numerator factor, exponential) so that
// flux = factor * (c_in * e - c_out).
template <class P, bool kCipa, int z>
__device__ __forceinline__ void ghk(double V, typename P::G v, typename P::G &fac, typename P::G &e) {
  using G = typename P::G;
  if constexpr (P::kMixed) {
    const G x = (G)z * v * (G)k::FRT;
    e = P::ex(x);
    fac = ghk_factor_e(x, e) * (G)k::F / (G)z;  // = vffrt / (e^{z vfrt} - 1)
  } else if constexpr (kCipa) {
    const double ffrt = k::F * k::FRT, B = (double)z * k::FRT;
    const double U = B * V;
    const double ee = exp_f64((double)z * (V * k::FRT));
    e = ee;
    // A*U/(e^U - 1) with A = ffrt*(...)/B  ->  factor = ffrt/B * U/(e^U - 1)
    fac = (-1.0e-07 <= U && U <= 1.0e-07) ? (ffrt / B) * (1.0 - 0.5 * U) : (ffrt / B) * div64(U, ee - 1.0);
  } else {
    const double vffrt = (V * k::F * k::F) / (k::R * k::T);
    const double ee = exp_f64((double)z * ((V * k::F) / (k::R * k::T)));
    e = ee;
    fac = div64(vffrt, ee - 1.0);
  }
}

// role 0: fast and late sodium, background sodium, Na/K pump; in FP64 the
// inward rectifier (kIK1InNa)
template <class P, bool kCipa>
__device__ __forceinline__ void role_na(Y<typename P::G> &y, const Par<typename P::G> &q, const Ctx<typename P::G> &c,
                                        double dt, bool update, Part<typename P::G> &o) {
  using G = typename P::G;
  const G v = c.v, one = (G)1;
  // the four logistic steady states of the group in one call
  const auto e_ss = P::grp4(-(v + (G)k::mssV1) * (G)(1.0 / k::mssV2), (v + (G)k::hssV1) * (G)(1.0 / k::hssV2),
                           -(v + (G)42.85) * (G)(1.0 / 5.264), (v + (G)87.61) * (G)(1.0 / 7.488));
  const G mss = P::rc((one + e_ss.a()));
  const Tau<P> tm = tau_quot<P>(1.0, (esum<P>((G)k::mtD1, (v + (G)k::mtV1) * (G)(1.0 / k::mtV2), (G)k::mtD2, -(v + (G)k::mtV3) * (G)(1.0 / k::mtV4))));
  const G e_hss = e_ss.b();
  const G hss = P::rc((one + e_hss));
  const Tau<P> thf = tau_quot<P>(1.0, (esum<P>((G)1.432e-05, -(v + (G)1.196) * (G)(1.0 / 6.285), (G)6.149, (v + (G)0.5096) * (G)(1.0 / 20.27))));
  const Tau<P> ths = tau_quot<P>(1.0, (esum<P>((G)0.009794, -(v + (G)17.95) * (G)(1.0 / 28.05), (G)0.3343, (v + (G)5.73) * (G)(1.0 / 56.66))));
  const Tau<P> tj = tau_affine<P>(2.038, (esum<P>((G)0.02136, -(v + (G)100.6) * (G)(1.0 / 8.281), (G)0.3052, (v + (G)0.9941) * (G)(1.0 / 38.45))));
  static_assert(k::hssV1 == 82.9 && k::hssV2 == 6.086, "hssp_shift assumes hss = 1/(1+e^((V+82.9)/6.086))");
  const G hssp = P::kFast ? P::rc(one + e_hss * (G)k::hssp_shift)
                           : P::rc((one + P::ex((v + (G)89.1) * (G)(1.0 / 6.086))));
  const G mLss = P::rc((one + e_ss.c()));
  const G e_hL = e_ss.d();
  const G hLss = P::rc((one + e_hL));
  const G hLssp = P::kFast ? P::rc(one + e_hL * (G)k::hLssp_shift)
                            : P::rc((one + P::ex((v + (G)93.81) * (G)(1.0 / 7.488))));
  const G fp_ = c.fCaMKp;
  // INa, INaL
  const G ENa = P::kFast ? (G)k::RTF * ((G)k::log_nao - P::lg((G)y.nai))
                          : (G)k::RTF * P::lg(P::dv((G)k::nao, (G)y.nai));
  const G h_ = (G)k::Ahf * (G)y.hf + (G)k::Ahs * (G)y.hs;
  const G hp = (G)k::Ahf * (G)y.hf + (G)k::Ahs * (G)y.hsp;
  const G INa = q.GNa * (v - ENa) * p3((G)y.m) * ((one - fp_) * h_ * (G)y.j + fp_ * hp * (G)y.jp);
  const G INaL = q.GNaL * (v - ENa) * (G)y.mL * ((one - fp_) * (G)y.hL + fp_ * (G)y.hLp);
  // INab
  G fac, e1;
  ghk<P, kCipa, 1>(y.V, v, fac, e1);
  const G INab = (G)k::PNab * fac * ((G)y.nai * e1 - (G)k::nao);
  // INaK
  const G nai_g = (G)y.nai, ki_g = (G)y.ki;
  // nao/Knao and nai/Knai: in mixed, nao/Knao0 e^(-c v) without a division
  G nao_Knao, nai_Knai;
  if constexpr (P::kFast) {
    const auto e_nak = P::grp2(-((one - (G)k::delta) * v * (G)k::F) * (G)(1.0 / (3.0 * k::R * k::T)),
                              -((G)k::delta * v * (G)k::F) * (G)(1.0 / (3.0 * k::R * k::T)));
    nao_Knao = (G)(k::nao / k::Knao0) * e_nak.a();
    nai_Knai = nai_g * (G)(1.0 / k::Knai0) * e_nak.b();
  } else {
    const G Knao = (G)k::Knao0 * P::ex(((one - (G)k::delta) * v * (G)k::F) * (G)(1.0 / (3.0 * k::R * k::T)));
    const G Knai = (G)k::Knai0 * P::ex(((G)k::delta * v * (G)k::F) * (G)(1.0 / (3.0 * k::R * k::T)));
    nao_Knao = P::dv((G)k::nao, Knao);
    nai_Knai = P::dv(nai_g, Knai);
  }
  const G nak_den_o = (p3(one + nao_Knao) + (G)k::ko_Kko_sq) - one;
  const G nak_den_i = (p3(one + nai_Knai) + p2(one + ki_g * (G)(1.0 / k::Kki))) - one;
  const G a3 = P::dv((G)k::a3c, nak_den_o);
  // P = eP / (1 + H/Khp + nai/Knap + ki/Kxkur) with the instance's H folded
  // into b3c = k3m*H/(1+MgATP/Kmgatp)
  const G H_Khp = q.b3c * (G)((1.0 + k::MgATP / k::Kmgatp) / (k::k3m * k::Khp));
  const G PP = P::dv((G)k::eP, (one + H_Khp + nai_g * (G)(1.0 / k::Knap) + ki_g * (G)(1.0 / k::Kxkur)));
  const G b3 = q.b3c * PP;
  const G a1 = P::dv(((G)k::k1p * p3(nai_Knai)), nak_den_i);
  const G b2 = P::dv(((G)k::k2m * p3(nao_Knao)), nak_den_o);
  const G b4 = P::dv(((G)k::k4m * p2(ki_g * (G)(1.0 / k::Kki))), nak_den_i);
  const G x1 = (G)k::a4 * a1 * (G)k::a2 + b2 * b4 * b3 + (G)k::a2 * b4 * b3 + b3 * a1 * (G)k::a2;
  const G x2 = b2 * (G)k::b1 * b4 + a1 * (G)k::a2 * a3 + a3 * (G)k::b1 * b4 + (G)k::a2 * a3 * b4;
  const G x3 = (G)k::a2 * a3 * (G)k::a4 + b3 * b2 * (G)k::b1 + b2 * (G)k::b1 * (G)k::a4 + a3 * (G)k::a4 * (G)k::b1;
  const G x4 = b4 * b3 * b2 + a3 * (G)k::a4 * a1 + b2 * (G)k::a4 * a1 + b3 * b2 * a1;
  const G xs_inv = P::rc((x1 + x2 + x3 + x4));
  const G JnakNa = (G)3.0 * (x1 * xs_inv * a3 - x2 * xs_inv * b3);
  const G JnakK = (G)2.0 * (x4 * xs_inv * (G)k::b1 - x3 * xs_inv * a1);
  const G INaK = q.Pnak * ((G)k::zna * JnakNa + (G)k::zk * JnakK);
  if constexpr (kIK1InNa<P>) {  // IK1 with its gate xk1 (see kIK1InNa)
    const auto e_k1 = P::grp2(-(v + (G)k::xk1_off) * (G)(1.0 / k::xk1_den),
                              ((v + (G)105.8) - (G)(2.6 * k::ko)) * (G)(1.0 / 9.493));
    const G xk1ss = P::rc((one + e_k1.a()));
    const Tau<P> txk1 =
        tau_quot<P>(122.2, (esum<P>((G)1, -(v + (G)127.2) * (G)(1.0 / 20.36), (G)1, (v + (G)236.8) * (G)(1.0 / 69.33))));
    const G EK = P::kFast ? (G)k::RTF * ((G)k::log_ko - P::lg((G)y.ki))
                           : (G)k::RTF * P::lg(P::dv((G)k::ko, (G)y.ki));
    const G rk1 = P::rc((one + e_k1.b()));
    const G IK1 = q.GK1 * (G)k::sqrt_ko * rk1 * (G)y.xk1 * (v - EK);
    o.f[S_iV] = INa + INaL + INaK + INab + IK1;
    o.f[S_iK] = IK1 - (G)2.0 * INaK;
    o.f[S_IK1] = IK1;
    if (update) y.xk1 = rush_larsen<P, true>(y.xk1, xk1ss, txk1, dt);
  } else {
    o.f[S_iV] = INa + INaL + INaK + INab;
    o.f[S_iK] = -(G)2.0 * INaK;
  }
  o.f[S_iNa] = INa + INaL + (G)3.0 * INaK + INab;
  o.f[S_INa] = INa;
  o.f[S_INaL] = INaL;
  if (!update) return;
  y.m = rush_larsen<P>(y.m, mss, tm, dt);
  y.hf = rush_larsen<P>(y.hf, hss, thf, dt);
  y.hs = rush_larsen<P, true>(y.hs, hss, ths, dt);
  y.j = rush_larsen<P, true>(y.j, hss, tj, dt);
  y.hsp = rush_larsen<P, true>(y.hsp, hssp, tau_scaled<P>(ths, 3.0), dt);
  y.jp = rush_larsen<P, true>(y.jp, hss, tau_scaled<P>(tj, 1.46), dt);
  y.mL = rush_larsen<P>(y.mL, mLss, tm, dt);
  y.hL = rush_larsen<P, true>(y.hL, hLss, tau_const<P>(k::thL), dt);
  y.hLp = rush_larsen<P, true>(y.hLp, hLssp, tau_const<P>(k::thLp), dt);
}

// role 1: transient outward, slow/rapid (ORd) delayed rectifier and
// background potassium currents, in the mixed path the inward rectifier
// (kIK1InNa); the stimulus
template <class P, bool kCipa>
__device__ __forceinline__ void role_k(Y<typename P::G> &y, const Par<typename P::G> &q, const Ctx<typename P::G> &c,
                                       double dt, bool update, Part<typename P::G> &o) {
  using G = typename P::G;
  const G v = c.v, one = (G)1;
  // the group's single exponentials, four per call
  const auto e_k1 = P::grp4(-(v - (G)14.34) * (G)(1.0 / 14.82), -(v - (G)18.4099) * (G)(1.0 / 29.3814),
                           (v + (G)100.0) * (G)(1.0 / 29.3814), (v + (G)43.94) * (G)(1.0 / 5.711));
  const auto e_k2 = P::grp4(-(v + (G)11.60) * (G)(1.0 / 8.932), -(v - (G)14.48) * (G)(1.0 / 18.34),
                           (v - (G)213.6) * (G)(1.0 / 151.2), (v + (G)70.0) * (G)0.05);
  const G e_a = e_k1.a();
  const G ass = P::rc((one + e_a));
  const Tau<P> ta = tau_quot<P>(1.0515, (P::rc(((G)1.2089 * (one + e_k1.b()))) + P::dv((G)3.5, (one + e_k1.c()))));
  const G assp = P::kFast ? P::rc(one + e_a * (G)k::assp_shift)
                           : P::rc((one + P::ex(-(v - (G)24.34) * (G)(1.0 / 14.82))));
  const G iss = P::rc((one + e_k1.d()));
  const G delta_epi = q.celltype == 1 ? one - P::dv((G)0.95, (one + P::ex((v + (G)70.0) * (G)0.2))) : one;
  const Tau<P> tiF = tau_affine<P>(4.562, (esum<P>((G)0.3933, -(v + (G)100.0) * (G)0.01, (G)0.08004, (v + (G)50.0) * (G)(1.0 / 16.59))), delta_epi);
  const Tau<P> tiS = tau_affine<P>(23.62, (esum<P>((G)0.001416, -(v + (G)96.52) * (G)(1.0 / 59.05), (G)1.78e-08, (v + (G)114.1) * (G)(1.0 / 8.079))), delta_epi);
  const G dti_develop = (G)1.354 + P::dv((G)1e-4, (esum<P>((G)1, (v - (G)167.4) * (G)(1.0 / 15.89), (G)1, -(v - (G)12.23) * (G)(1.0 / 0.2154))));
  const G dti_recover = one - P::dv((G)0.5, (one + e_k2.d()));
  const G dti = dti_develop * dti_recover;
  const G xs1ss = P::rc((one + e_k2.a()));
  const Tau<P> txs1 = tau_affine<P>(817.3, (esum<P>((G)2.326e-04, (v + (G)48.28) * (G)(1.0 / 17.80), (G)0.001292, -(v + (G)210.0) * (G)(1.0 / 230.0))));
  const Tau<P> txs2 =
      tau_quot<P>(1.0, (esum<P>((G)0.01, (v - (G)50.0) * (G)0.05, (G)0.0193, -(v + (G)66.54) * (G)(1.0 / 31.0))));
  const G fp_ = c.fCaMKp;
  const G EK = P::kFast ? (G)k::RTF * ((G)k::log_ko - P::lg((G)y.ki))
                         : (G)k::RTF * P::lg(P::dv((G)k::ko, (G)y.ki));
  const G AiF = P::rc((one + e_k2.c()));
  const G AiS = one - AiF;
  const G i_ = AiF * (G)y.iF + AiS * (G)y.iS;
  const G ip = AiF * (G)y.iFp + AiS * (G)y.iSp;
  const G Ito = q.Gto * (v - EK) * ((one - fp_) * (G)y.a * i_ + fp_ * (G)y.ap * ip);
  G IKr = (G)0, xrss = (G)0;
  Tau<P> txrf = tau_const<P>(1.0), txrs = tau_const<P>(1.0);
  if constexpr (!kCipa) {
    const auto e_kr = P::grp4(-(v + (G)8.337) * (G)(1.0 / 6.789), (v + (G)54.81) * (G)(1.0 / 38.21),
                             (v + (G)55.0) * (G)(1.0 / 75.0), (v - (G)10.0) * (G)(1.0 / 30.0));
    xrss = P::rc((one + e_kr.a()));
    txrf = tau_affine<P>(12.98, (esum<P>((G)0.3652, (v - (G)31.66) * (G)(1.0 / 3.869), (G)4.123e-05, -(v - (G)47.78) * (G)(1.0 / 20.38))));
    txrs = tau_affine<P>(1.865, (esum<P>((G)0.06629, (v - (G)34.70) * (G)(1.0 / 7.355), (G)1.128e-05, -(v - (G)29.74) * (G)(1.0 / 25.94))));
    const G Axrf = P::rc((one + e_kr.b()));
    const G xr = Axrf * (G)y.xrf + (one - Axrf) * (G)y.xrs;
    const G rkr = P::kFast ? P::rc((one + e_kr.c()) * (one + e_kr.d()))
                            : P::dv((P::rc((one + e_kr.c()))), (one + e_kr.d()));
    IKr = q.GKr * (G)k::sqrt_ko54 * xr * rkr * (v - EK);
  }
  const G EKs = P::kFast
                    ? (G)k::RTF * ((G)k::log_ks_o - P::lg((G)(y.ki + k::PKNa * y.nai)))
                    : (G)k::RTF * P::lg(P::dv((G)(k::ko + k::PKNa * k::nao), (G)(y.ki + k::PKNa * y.nai)));
  const G KsCa = P::kFast
                     ? one + P::dv((G)0.6, (one + P::ex((G)1.4 * ((G)k::log_ks_ca - P::lg((G)y.cai)))))
                     : one + P::dv((G)0.6, (one + P::pw(P::dv((G)3.8e-05, (G)y.cai), (G)1.4)));
  const G IKs = q.GKs * KsCa * (G)y.xs1 * (G)y.xs2 * (v - EKs);
  const G xkb = P::rc((one + e_k2.b()));
  const G IKb = q.GKb * xkb * (v - EK);
  const G Istim = c.stim ? (G)q.amp : (G)0;
  G IK1 = (G)0, xk1ss = (G)0;
  Tau<P> txk1 = tau_const<P>(1.0);
  if constexpr (!kIK1InNa<P>) {  // IK1 with its gate xk1 (see kIK1InNa)
    const auto e_ik1 = P::grp2(-(v + (G)k::xk1_off) * (G)(1.0 / k::xk1_den),
                               ((v + (G)105.8) - (G)(2.6 * k::ko)) * (G)(1.0 / 9.493));
    xk1ss = P::rc((one + e_ik1.a()));
    txk1 = tau_quot<P>(122.2, (esum<P>((G)1, -(v + (G)127.2) * (G)(1.0 / 20.36), (G)1, (v + (G)236.8) * (G)(1.0 / 69.33))));
    IK1 = q.GK1 * (G)k::sqrt_ko * P::rc((one + e_ik1.b())) * (G)y.xk1 * (v - EK);
    o.f[S_IK1] = IK1;
  }
  o.f[S_iV] = Ito + IKr + IKs + IK1 + IKb + Istim;
  o.f[S_iK] = Ito + IKr + IKs + IK1 + IKb + Istim;
  o.f[S_Ito] = Ito;
  o.f[S_IKr] = IKr;
  o.f[S_IKs] = IKs;
  if (!update) return;
  if constexpr (!kIK1InNa<P>) y.xk1 = rush_larsen<P, true>(y.xk1, xk1ss, txk1, dt);
  y.a = rush_larsen<P, true>(y.a, ass, ta, dt);
  y.iF = rush_larsen<P, true>(y.iF, iss, tiF, dt);
  y.iS = rush_larsen<P, true>(y.iS, iss, tiS, dt);
  y.ap = rush_larsen<P, true>(y.ap, assp, ta, dt);
  y.iFp = rush_larsen<P, true>(y.iFp, iss, tau_times<P>(tiF, dti), dt);
  y.iSp = rush_larsen<P, true>(y.iSp, iss, tau_times<P>(tiS, dti), dt);
  y.xs1 = rush_larsen<P, true>(y.xs1, xs1ss, txs1, dt);
  y.xs2 = rush_larsen<P, true>(y.xs2, xs1ss, txs2, dt);
  if constexpr (!kCipa) {
    y.xrf = rush_larsen<P, true>(y.xrf, xrss, txrf, dt);
    y.xrs = rush_larsen<P, true>(y.xrs, xrss, txrs, dt);
  }
}

// role 2: L-type calcium channel (Ca, Na, K components), background and
// pump calcium currents, ryanodine-receptor release
template <class P, bool kCipa>
__device__ __forceinline__ void role_ca(Y<typename P::G> &y, const Par<typename P::G> &q, const Ctx<typename P::G> &c,
                                        double dt, bool update, Part<typename P::G> &o) {
  using G = typename P::G;
  const G v = c.v, one = (G)1;
  const auto e_ca = P::grp2(-(v + (G)3.94) * (G)(1.0 / 4.23), (v + (G)19.58) * (G)(1.0 / 3.696));
  const G dss = P::rc((one + e_ca.a()));
  const Tau<P> td = tau_affine<P>(0.6, (esum<P>((G)1, (G)-0.05 * (v + (G)6.0), (G)1, (G)0.09 * (v + (G)14.0))));
  const G fss = P::rc((one + e_ca.b()));
  const Tau<P> tff = tau_affine<P>(7.0, (esum<P>((G)0.0045, -(v + (G)20.0) * (G)0.1, (G)0.0045, (v + (G)20.0) * (G)0.1)));
  const Tau<P> tfs = tau_affine<P>(1000.0, (esum<P>((G)3.5e-05, -(v + (G)5.0) * (G)0.25, (G)3.5e-05, (v + (G)5.0) * (G)(1.0 / 6.0))));
  const Tau<P> tfcaf = tau_affine<P>(7.0, (esum<P>((G)0.04, -(v - (G)4.0) * (G)(1.0 / 7.0), (G)0.04, (v - (G)4.0) * (G)(1.0 / 7.0))));
  const Tau<P> tfcas = tau_affine<P>(100.0, (esum<P>((G)0.00012, -v * (G)(1.0 / 3.0), (G)0.00012, v * (G)(1.0 / 7.0))));
  const G km2n = (G)y.jca;
  const G cass_g = (G)y.cass, cai_g = (G)y.cai, cajsr_g = (G)y.cajsr;
  const G anca = P::rc((P::dv((G)k::k2n, km2n) + p4(one + P::dv((G)k::Kmn, cass_g))));
  const G f = q.Aff * (G)y.ff + q.Afs * (G)y.fs;
  const G Afcaf = (G)0.3 + P::dv((G)0.6, (one + P::ex((v - (G)10.0) * (G)0.1)));
  const G Afcas = one - Afcaf;
  const G fca = Afcaf * (G)y.fcaf + Afcas * (G)y.fcas;
  const G fp = q.Aff * (G)y.ffp + q.Afs * (G)y.fs;
  const G fcap = Afcaf * (G)y.fcafp + Afcas * (G)y.fcas;
  const G fICaLp = c.fCaMKp;
  const G nca_ = (G)y.nca, jca_ = (G)y.jca, d_ = (G)y.d;
  const G gate_np = d_ * (f * (one - nca_) + jca_ * fca * nca_);
  const G gate_p = d_ * (fp * (one - nca_) + jca_ * fcap * nca_);
  G fac1, e1, fac2, e2;
  ghk<P, kCipa, 1>(y.V, v, fac1, e1);
  if constexpr (P::kMixed) {  // e^{2x} = (e^x)^2
    const G x2 = (G)2 * v * (G)k::FRT;
    e2 = e1 * e1;
    fac2 = ghk_factor_e(x2, e2) * (G)k::F / (G)2;
  } else {
    ghk<P, kCipa, 2>(y.V, v, fac2, e2);
  }
  const G PhiCaL = (G)4.0 * fac2 * (cass_g * e2 - (G)(0.341 * k::cao));
  const G PhiCaNa = fac1 * ((G)0.75 * (G)y.nass * e1 - (G)(0.75 * k::nao));
  const G PhiCaK = fac1 * ((G)0.75 * (G)y.kss * e1 - (G)(0.75 * k::ko));
  const G ICab = (G)(k::PCab * 4.0) * fac2 * (cai_g * e2 - (G)(0.341 * k::cao));
  const G ICaL = (one - fICaLp) * q.PCa * PhiCaL * gate_np + fICaLp * q.PCap * PhiCaL * gate_p;
  const G ICaNa = (one - fICaLp) * q.PCaNa * PhiCaNa * gate_np + fICaLp * q.PCaNap * PhiCaNa * gate_p;
  const G ICaK = (one - fICaLp) * q.PCaK * PhiCaK * gate_np + fICaLp * q.PCaKp * PhiCaK * gate_p;
  const G IpCa = P::dv(((G)k::GpCa * cai_g), ((G)k::KmCap + cai_g));
  const G Jrel = (one - fICaLp) * (G)y.Jrelnp + fICaLp * (G)y.Jrelp;
  o.f[S_iV] = ICaL + ICaNa + ICaK + IpCa + ICab;
  o.f[S_iNass] = ICaNa;
  o.f[S_iKss] = ICaK;
  o.f[S_iCass] = ICaL;
  o.f[S_iCai] = IpCa + ICab;
  o.f[S_Jrel] = Jrel;
  o.f[S_ICaL] = ICaL;
  if (!update) return;
  const G rel_den = one + p8(P::dv((G)1.5, cajsr_g));
  const G den_tau = one + P::dv((G)0.0123, cajsr_g);
  G Jrel_inf_t, Jrel_t;
  Tau<P> tau_rel, tau_relp;  // bt / den_tau, floored at 0.001 ms
  if constexpr (P::kFast) {  // one reciprocal for both targets; rates capped at 1000 /ms
    const G r = P::rc(rel_den);
    Jrel_inf_t = (G)k::a_rel * -ICaL * r;
    Jrel_t = (G)k::a_relp * -ICaL * r;
    // the floor also catches a negative tau (cajsr briefly below -0.0123
    // under forward Euler): bt / den_tau < 0.001 holds for den_tau < 0 too,
    // so a negative rate takes the cap, as the written form does
    const G r1 = den_tau * (G)(1.0 / k::bt), r2 = den_tau * (G)(1.0 / k::btp);
    tau_rel = Tau<P>{(r1 > (G)1000 || r1 < (G)0) ? (G)1000 : r1};
    tau_relp = Tau<P>{(r2 > (G)1000 || r2 < (G)0) ? (G)1000 : r2};
  } else {
    Jrel_inf_t = P::dv(((G)k::a_rel * -ICaL), rel_den);
    Jrel_t = P::dv(((G)k::a_relp * -ICaL), rel_den);
    const G t1 = P::dv((G)k::bt, den_tau), t2 = P::dv((G)k::btp, den_tau);
    tau_rel = Tau<P>{t1 < (G)0.001 ? (G)0.001 : t1};
    tau_relp = Tau<P>{t2 < (G)0.001 ? (G)0.001 : t2};
  }
  const G Jrel_inf = q.celltype == 2 ? Jrel_inf_t * (G)1.7 : Jrel_inf_t;
  const G Jrel_infp = q.celltype == 2 ? Jrel_t * (G)1.7 : Jrel_t;
  y.d = rush_larsen<P, true>(y.d, dss, td, dt);
  y.ff = rush_larsen<P, true>(y.ff, fss, tff, dt);
  y.fs = rush_larsen<P, true>(y.fs, fss, tfs, dt);
  y.fcaf = rush_larsen<P, true>(y.fcaf, fss, tfcaf, dt);
  y.fcas = rush_larsen<P, true>(y.fcas, fss, tfcas, dt);
  y.jca = rush_larsen<P, true>(y.jca, fss, q.tjca, dt);
  y.ffp = rush_larsen<P, true>(y.ffp, fss, tau_scaled<P>(tff, 2.5), dt);
  // quirk (1): the reference steps fcafp by d = 25 (exp(-25/tfcafp)), far
  // outside the Taylor range, so that case takes the exponential form
  if (q.fcafp_dt != (G)0)
    y.fcafp = rush_larsen<P>(y.fcafp, fss, tau_scaled<P>(tfcaf, 2.5), (double)q.fcafp_dt);
  else
    y.fcafp = rush_larsen<P, true>(y.fcafp, fss, tau_scaled<P>(tfcaf, 2.5), dt);
  // nca relaxes at rate km2n towards anca*k2n/km2n (Ohara_Rudy_2011.cpp:1065-1066)
  y.nca = rush_larsen<P, true>(y.nca, anca * P::dv((G)k::k2n, km2n), tau_quot<P>(1.0, km2n), dt);
  y.Jrelnp = rush_larsen<P>(y.Jrelnp, Jrel_inf, tau_rel, dt);
  y.Jrelp = rush_larsen<P>(y.Jrelp, Jrel_infp, tau_relp, dt);
}

// Na/Ca exchanger current of one compartment (INaCa_i or INaCa_ss, the
// 0.8/0.2 split of Ohara_Rudy_2011.cpp:923-958); na, ca: the compartment's
// concentrations; hna, hca, h8, k3pp, k8, k3: the voltage-only factors.
template <class P>
__device__ __forceinline__ typename P::G naca(typename P::G na, typename P::G ca, typename P::G hna,
                                              typename P::G hca, typename P::G h8, typename P::G k3pp,
                                              typename P::G k8, typename P::G k3, typename P::G Gncx,
                                              typename P::G split) {
  using G = typename P::G;
  const G one = (G)1;
  const G h1 = one + ((na) * (G)(1.0 / k::kna3)) * (one + hna);
  const G h4 = one + ((na) * (G)(1.0 / k::kna1)) * (one + (na) * (G)(1.0 / k::kna2));
  G h2, h5, k4p, k6;
  if constexpr (P::kFast) {  // 1/h1, 1/h4 (and 1/hca, shared by both compartments) each once
    const G rh1 = P::rc(h1), rh4 = P::rc(h4);
    h2 = na * hna * (G)(1.0 / k::kna3) * rh1;
    h5 = na * na * (G)(1.0 / (k::kna1 * k::kna2)) * rh4;
    k4p = rh1 * (G)k::wca * P::rc(hca);
    k6 = rh4 * ca * (G)k::kcaon;
  } else {
    h2 = P::dv((na * hna), ((G)k::kna3 * h1));
    h5 = P::dv((na * na), (h4 * (G)k::kna1 * (G)k::kna2));
    k4p = P::dv(((P::rc(h1)) * (G)k::wca), hca);
    k6 = (P::rc(h4)) * ca * (G)k::kcaon;
  }
  const G k4pp = h2 * (G)k::wnaca;
  const G k7 = h5 * h2 * (G)k::wna;
  const G k4 = k4p + k4pp;
  const G x1 = (G)k::k2x * k4 * (k7 + k6) + (G)k::k5x * k7 * ((G)k::k2x + k3);
  const G x2 = (G)k::k1x * k7 * (k4 + (G)k::k5x) + k4 * k6 * ((G)k::k1x + k8);
  const G x3 = (G)k::k1x * k3 * (k7 + k6) + k8 * k6 * ((G)k::k2x + k3);
  const G x4 = (G)k::k2x * k8 * (k4 + (G)k::k5x) + k3 * (G)k::k5x * ((G)k::k1x + k8);
  const G inv = P::rc((x1 + x2 + x3 + x4));
  const G allo = P::rc((one + p2(P::dv((G)k::KmCaAct, ca))));
  const G JncxNa = ((G)3.0 * (x4 * inv * k7 - x1 * inv * k8) + x3 * inv * k4pp) - x2 * inv * k3pp;
  const G JncxCa = x2 * inv * (G)k::k2x - x1 * inv * (G)k::k1x;
  return split * Gncx * allo * ((G)k::zna * JncxNa + (G)k::zca * JncxCa);
}

// role 3: Na/Ca exchange (both compartments), SERCA uptake; CiPA: the
// dynamic hERG Markov chain with drug binding/trapping and IKr
// One backward-Euler step of the CiPA Markov IKr chain with the rates
// frozen at the step's V: (I - h Q) x = g, g = h Q S (the forward-Euler
// increments, in place in g on entry, x on return), states in the order
// IC1, IC2, C1, C2, O, IO, IObound, Obound, Cbound; k = {k11, k21, k51,
// k61, k3, k4, k52, k62, k1, k2, k31, k41, k53, k63, bind, Ku, unb, trap,
// Kt}. The sparse system is eliminated in a fixed order (Cb; the bound pair
// as affine functions of O and IO; IC1; C1; C2; the dense 3x3 IC2, O, IO)
// with no pivoting (I - h Q is an M-matrix); total occupancy is kept.
template <class P>
__device__ __forceinline__ void markov_be(typename P::G h, const typename P::G *k, typename P::G *g) {
  using G = typename P::G;
  const G one = (G)1;
  const G k11 = k[0], k21 = k[1], k51 = k[2], k61 = k[3], k3 = k[4], k4 = k[5], k52 = k[6], k62 = k[7];
  const G k1 = k[8], k2 = k[9], k31 = k[10], k41 = k[11], k53 = k[12], k63 = k[13], bind = k[14];
  const G Ku = k[15], unb = k[16], trap = k[17], Kt = k[18];
  const G dIC1 = one + h * (k11 + k61), dIC2 = one + h * ((k21 + k3) + k62), dC1 = one + h * (k51 + k1);
  const G dC2 = one + h * ((k2 + k52) + k31), dO = one + h * ((k41 + k53) + bind);
  const G dIO = one + h * ((k4 + k63) + bind), dIOb = one + h * (unb + Kt), dOb = one + h * (Ku + Kt);
  const G rCb = P::rc(one + h * ((G)2 * trap));
  const G ht = h * trap, hK = h * Kt, hb = h * bind;
  const G c = ht * hK * rCb, e = ht * g[8] * rCb;
  const G a11 = dOb - c, a22 = dIOb - c, rdet = P::rc(a11 * a22 - c * c);
  const G rOb = g[7] + e, rIOb = g[6] + e;
  const G ob0 = (a22 * rOb + c * rIOb) * rdet, obO = a22 * hb * rdet, obIO = c * hb * rdet;
  const G iob0 = (c * rOb + a11 * rIOb) * rdet, iobO = c * hb * rdet, iobIO = a11 * hb * rdet;
  const G aOO = dO - h * Ku * obO, aOIO = -(h * k63 + h * Ku * obIO), aOC2 = -h * k31;
  const G rO = g[4] + h * Ku * ob0;
  const G aIOIO = dIO - h * unb * iobIO, aIOO = -(h * k53 + h * unb * iobO), aIOIC2 = -h * k3;
  const G rIO = g[5] + h * unb * iob0;
  const G rIC1 = P::rc(dIC1);
  const G i0 = g[0] * rIC1, iI2 = h * k21 * rIC1, iC1 = h * k51 * rIC1;
  const G re11 = P::rc(dC1 - h * k61 * iC1);
  const G c0 = (g[2] + h * k61 * i0) * re11, cI2 = h * k61 * iI2 * re11, cC2 = h * k2 * re11;
  const G bII = dIC2 - h * k11 * (iI2 + iC1 * cI2), bIC = -(h * k52 + h * k11 * iC1 * cC2);
  const G bIIO = -h * k4, rI = g[1] + h * k11 * (i0 + iC1 * c0);
  const G rCC = P::rc(dC2 - h * k1 * cC2), bCI = -(h * k62 + h * k1 * cI2), bCO = -h * k41;
  const G rC = g[3] + h * k1 * c0;
  const G m11 = bII - bIC * bCI * rCC, m12 = -bIC * bCO * rCC, m13 = bIIO, s1 = rI - bIC * rC * rCC;
  const G m21 = -aOC2 * bCI * rCC, m22 = aOO - aOC2 * bCO * rCC, m23 = aOIO, s2 = rO - aOC2 * rC * rCC;
  const G m31 = aIOIC2, m32 = aIOO, m33 = aIOIO, s3 = rIO;
  const G r11 = P::rc(m11);
  const G l21 = m21 * r11, l31 = m31 * r11;
  const G n22 = m22 - l21 * m12, n23 = m23 - l21 * m13, t2 = s2 - l21 * s1;
  const G n32 = m32 - l31 * m12, n33 = m33 - l31 * m13, t3 = s3 - l31 * s1;
  const G r22 = P::rc(n22);
  const G l32 = n32 * r22;
  const G xIO = P::dv(t3 - l32 * t2, n33 - l32 * n23);
  const G xO = (t2 - n23 * xIO) * r22;
  const G xIC2 = ((s1 - m12 * xO) - m13 * xIO) * r11;
  const G xC2 = ((rC - bCI * xIC2) - bCO * xO) * rCC;
  const G xC1 = (c0 + cI2 * xIC2) + cC2 * xC2;
  const G xOb = (ob0 + obO * xO) + obIO * xIO, xIOb = (iob0 + iobO * xO) + iobIO * xIO;
  g[8] = (g[8] + hK * (xIOb + xOb)) * rCb;
  g[0] = (i0 + iI2 * xIC2) + iC1 * xC1;
  g[1] = xIC2; g[2] = xC1; g[3] = xC2; g[4] = xO; g[5] = xIO; g[6] = xIOb; g[7] = xOb;
}

template <class P, bool kCipa>
__device__ __forceinline__ void role_x(Y<typename P::G> &y, const Par<typename P::G> &q, const Ctx<typename P::G> &c,
                                       double dt, bool update, Part<typename P::G> &o) {
  using G = typename P::G;
  const G v = c.v, one = (G)1;
  const auto e_x = P::grp2(((G)k::qna * v) * (G)k::FRT, ((G)k::qca * v) * (G)k::FRT);
  const G hna = e_x.a();
  const G hca = e_x.b();
  const G h7 = one + ((G)k::nao / (G)k::kna3) * (one + P::rc(hna));
  const G h8 = P::dv((G)k::nao, ((G)k::kna3 * hna * h7));
  const G k3pp = h8 * (G)k::wnaca;
  const G k8 = h8 * (G)k::h11 * (G)k::wna;
  const G k3 = (P::rc(h7)) * (G)k::wca + k3pp;
  const G cai_g = (G)y.cai;
  const G INaCa_i = naca<P>((G)y.nai, cai_g, hna, hca, h8, k3pp, k8, k3, q.Gncx, (G)0.8);
  const G INaCa_ss = naca<P>((G)y.nass, (G)y.cass, hna, hca, h8, k3pp, k8, k3, q.Gncx, (G)0.2);
  const G fp_ = c.fCaMKp;
  const G Jupnp = P::dv((q.upScale * (G)0.004375 * cai_g), (cai_g + (G)0.00092));
  const G Jupp = P::dv((q.upScale * (G)(2.75 * 0.004375) * cai_g), ((cai_g + (G)0.00092) - (G)0.00017));
  const G Jleak = (G)(0.0039375 / 15.0) * (G)y.cansr;
  const G Jup = ((one - fp_) * Jupnp + fp_ * Jupp) - Jleak;
  G IKr = (G)0;
  if constexpr (kCipa) {
    // dynamic hERG: IKr = GKr sqrt(ko/5.4) O (V - EK) (ohara_rudy_cipa_v1_2017.cpp:2307)
    const G EK = P::kFast ? (G)k::RTF * ((G)k::log_ko - P::lg((G)y.ki))
                           : (G)k::RTF * P::lg(P::dv((G)k::ko, (G)y.ki));
    IKr = q.GKr * (G)k::sqrt_ko54 * (G)y.O * (v - EK);
  }
  o.f[S_iV] = INaCa_i + INaCa_ss + IKr;
  o.f[S_iNa] = (G)3.0 * INaCa_i;
  o.f[S_iNass] = (G)3.0 * INaCa_ss;
  o.f[S_iCass] = -(G)2.0 * INaCa_ss;
  o.f[S_iCai] = -(G)2.0 * INaCa_i;
  o.f[S_Jup] = Jup;
  o.f[S_IKr] = IKr;
  o.f[S_iK] = IKr;  // CiPA's IKr is a potassium flux too (zero for ORd: role 1 carries it)
  if constexpr (kCipa) {
    if (!update) return;
    // Markov IKr with drug binding and trapping (ohara_rudy_cipa_v1_2017.cpp:
    // 2157-2165), forward Euler like every other non-gate state. Rates
    // k = A exp(B V) Q10; bound-drug states use the instance's bind = Kmax Ku
    // D^n/(D^n + halfmax), Ku, and Kt / (1 + exp(-(V - Vhalf)/6.789)).
    const auto e1_2 = P::ex2((G)cipa::B1 * v, (G)cipa::B2 * v);
    const G k1 = (G)cipa::A1 * e1_2.a * (G)cipa::Q1;
    const G k2 = (G)cipa::A2 * e1_2.b * (G)cipa::Q2;
    const auto e3_4 = P::ex2((G)cipa::B3 * v, (G)cipa::B4 * v);
    const G k3m = (G)cipa::A3 * e3_4.a * (G)cipa::Q3;
    const G k4m = (G)cipa::A4 * e3_4.b * (G)cipa::Q4;
    const auto e11_21 = P::ex2((G)cipa::B11 * v, (G)cipa::B21 * v);
    const G k11 = (G)cipa::A11 * e11_21.a * (G)cipa::Q11;
    const G k21 = (G)cipa::A21 * e11_21.b * (G)cipa::Q21;
    const auto e31_41 = P::ex2((G)cipa::B31 * v, (G)cipa::B41 * v);
    const G k31 = (G)cipa::A31 * e31_41.a * (G)cipa::Q31;
    const G k41 = (G)cipa::A41 * e31_41.b * (G)cipa::Q41;
    const auto e51_52 = P::ex2((G)cipa::B51 * v, (G)cipa::B52 * v);
    const G k51 = (G)cipa::A51 * e51_52.a * (G)cipa::Q51;
    const G k52 = (G)cipa::A52 * e51_52.b * (G)cipa::Q52;
    const auto e53_61 = P::ex2((G)cipa::B53 * v, (G)cipa::B61 * v);
    const G k53 = (G)cipa::A53 * e53_61.a * (G)cipa::Q53;
    const G k61 = (G)cipa::A61 * e53_61.b * (G)cipa::Q61;
    const auto e62_63 = P::ex2((G)cipa::B62 * v, (G)cipa::B63 * v);
    const G k62 = (G)cipa::A62 * e62_63.a * (G)cipa::Q62;
    const G k63 = (G)cipa::A63 * e62_63.b * (G)cipa::Q63;
    const G unb = P::dv(q.Ku * k53, k63);
    const G trap = P::dv(q.Kt, one + P::ex(-(v - q.Vhalf) * (G)(1.0 / 6.789)));
    // The chain is linear in its states for this step's V: forward Euler
    // (the reference scheme for non-gate states) unless its largest outflow
    // rate makes that step unsafe (dt*lam > 1.8: fast drug binding, the
    // IC2 -> IC1 rate below ~-95 mV, IC1 -> C1 above ~43 mV); then one
    // backward-Euler step of the chain (markov_be), stable for any rate.
    G lam = k11 + k61;
    lam = fmax(lam, k21 + k3m + k62);
    lam = fmax(lam, k1 + k51);
    lam = fmax(lam, k2 + k31 + k52);
    lam = fmax(lam, k41 + k53 + q.bind);
    lam = fmax(lam, k4m + k63 + q.bind);
    lam = fmax(lam, unb + q.Kt);
    lam = fmax(lam, q.Ku + q.Kt);
    lam = fmax(lam, (G)2 * trap);
    const G IC1 = (G)y.IC1, IC2 = (G)y.IC2, C1 = (G)y.C1, C2 = (G)y.C2, O = (G)y.O, IO = (G)y.IO;
    const G IOb = (G)y.IObound, Ob = (G)y.Obound, Cb = (G)y.Cbound;
    const G f11 = k11 * IC1 - k21 * IC2, f51 = k51 * C1 - k61 * IC1, f3 = k3m * IC2 - k4m * IO;
    const G f52 = k52 * C2 - k62 * IC2, f1 = k1 * C1 - k2 * C2, f31 = k31 * C2 - k41 * O;
    const G f53 = k53 * O - k63 * IO, fbo = q.bind * O - q.Ku * Ob, fbi = q.bind * IO - unb * IOb;
    const G ftc = trap * Cb;
    G d[9] = {-f11 + f51, (f11 - f3) + f52, -f1 - f51, (f1 - f31) - f52, (f31 - f53) - fbo, (f3 + f53) - fbi,
              (fbi + ftc) - q.Kt * IOb, (fbo + ftc) - q.Kt * Ob, -(ftc - q.Kt * Ob) - (ftc - q.Kt * IOb)};
    if constexpr (P::kRates) {  // the chain's right-hand side
      y.IC1 = (double)d[0]; y.IC2 = (double)d[1]; y.C1 = (double)d[2]; y.C2 = (double)d[3]; y.O = (double)d[4];
      y.IO = (double)d[5]; y.IObound = (double)d[6]; y.Obound = (double)d[7]; y.Cbound = (double)d[8];
    } else if ((G)dt * lam > (G)1.8) {
      const G hh = (G)dt;
#pragma unroll
      for (int s = 0; s < 9; ++s) d[s] *= hh;
      const G kr[19] = {k11, k21, k51, k61, k3m, k4m, k52, k62, k1, k2, k31, k41, k53, k63, q.bind, q.Ku, unb, trap, q.Kt};
      markov_be<P>(hh, kr, d);
      y.IC1 += (double)d[0]; y.IC2 += (double)d[1]; y.C1 += (double)d[2]; y.C2 += (double)d[3];
      y.O += (double)d[4]; y.IO += (double)d[5]; y.IObound += (double)d[6]; y.Obound += (double)d[7];
      y.Cbound += (double)d[8];
    } else {
      y.IC1 += (double)d[0] * dt; y.IC2 += (double)d[1] * dt; y.C1 += (double)d[2] * dt;
      y.C2 += (double)d[3] * dt; y.O += (double)d[4] * dt; y.IO += (double)d[5] * dt;
      y.IObound += (double)d[6] * dt; y.Obound += (double)d[7] * dt; y.Cbound += (double)d[8] * dt;
    }
  }
}

template <class P, bool kCipa, int R>
__device__ __forceinline__ void role(Y<typename P::G> &y, const Par<typename P::G> &q, const Ctx<typename P::G> &c,
                                     double dt, bool update, Part<typename P::G> &o) {
  if constexpr (R == 0) role_na<P, kCipa>(y, q, c, dt, update, o);
  if constexpr (R == 1) role_k<P, kCipa>(y, q, c, dt, update, o);
  if constexpr (R == 2) role_ca<P, kCipa>(y, q, c, dt, update, o);
  if constexpr (R == 3) role_x<P, kCipa>(y, q, c, dt, update, o);
}

// Sum of the four roles' contributions, in role order (both kernels).
template <bool kIK1Na, class G>
__device__ __forceinline__ void add_part(Part<G> &s, const Part<G> &p, int role) {
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const int f = role_field<kIK1Na>(role, k);
    if (f >= 0) s.f[f] += p.f[f];
  }
}

// Forward Euler of V, ions and CaMKII from the summed contributions
// (Ohara_Rudy_2011.cpp:1082-1093); concentration differences are formed in
// FP64 before rounding. `cur` receives the currents and RATES[V].
template <class P>
__device__ __forceinline__ void combine(Y<typename P::G> &y, const Par<typename P::G> &q, const Part<typename P::G> &s,
                                        double dt, bool update, Cur<typename P::G> &cur) {
  using G = typename P::G;
  const G one = (G)1;
  const G dV = -s.f[S_iV];
  cur.INa = s.f[S_INa]; cur.INaL = s.f[S_INaL]; cur.ICaL = s.f[S_ICaL]; cur.Ito = s.f[S_Ito];
  cur.IKr = s.f[S_IKr]; cur.IKs = s.f[S_IKs]; cur.IK1 = s.f[S_IK1]; cur.dVdt = dV;
  if (!update) return;
  const G cass_g = (G)y.cass, cai_g = (G)y.cai, cajsr_g = (G)y.cajsr;
  const G JdiffK = (G)((y.kss - y.ki) * 0.5);
  const G JdiffNa = (G)((y.nass - y.nai) * 0.5);
  const G Jdiff = (G)((y.cass - y.cai) * 5.0);
  const G Jtr = (G)((y.cansr - y.cajsr) * 0.01);
  const G Bcass = P::rc((one + P::dv((G)(k::BSRmax * k::KmBSR), p2((G)k::KmBSR + cass_g)) +
                         P::dv((G)(k::BSLmax * k::KmBSL), p2((G)k::KmBSL + cass_g))));
  const G Bcai = P::rc((one + P::dv((q.cmdnmax * (G)k::kmcmdn), p2((G)k::kmcmdn + cai_g)) +
                        P::dv((G)(k::trpnmax * k::kmtrpn), p2((G)k::kmtrpn + cai_g))));
  const G Bcajsr = P::rc((one + P::dv((G)(k::csqnmax * k::kmcsqn), p2((G)k::kmcsqn + cajsr_g))));
  const double CaMKb = P::dv((k::CaMKo * (1.0 - y.CaMKt)), (1.0 + P::dv(k::KmCaM, y.cass)));
  const double dCaMKt = k::aCaMK * CaMKb * (CaMKb + y.CaMKt) - k::bCaMK * y.CaMKt;
  const G dki = (-s.f[S_iK]) * (G)k::cAF_myo + JdiffK * (G)(k::vss / k::vmyo);
  const G dkss = (-s.f[S_iKss]) * (G)k::cAF_ss - JdiffK;
  const G dnai = (-s.f[S_iNa]) * (G)k::cAF_myo + JdiffNa * (G)(k::vss / k::vmyo);
  const G dnass = (-s.f[S_iNass]) * (G)k::cAF_ss - JdiffNa;
  const G dcass = Bcass * (((-s.f[S_iCass]) * (G)(0.5 * k::cAF_ss) + s.f[S_Jrel] * (G)(k::vjsr / k::vss)) - Jdiff);
  const G dcai = Bcai * (((-s.f[S_iCai]) * (G)(0.5 * k::cAF_myo) - s.f[S_Jup] * (G)(k::vnsr / k::vmyo)) +
                         Jdiff * (G)(k::vss / k::vmyo));
  const G dcansr = s.f[S_Jup] - Jtr * (G)(k::vjsr / k::vnsr);
  const G dcajsr = Bcajsr * (Jtr - s.f[S_Jrel]);
  fe<P>(y.CaMKt, dCaMKt, dt);
  fe<P>(y.V, (double)dV, dt);
  fe<P>(y.nai, (double)dnai, dt);
  fe<P>(y.nass, (double)dnass, dt);
  fe<P>(y.ki, (double)dki, dt);
  fe<P>(y.kss, (double)dkss, dt);
  fe<P>(y.cai, (double)dcai, dt);
  fe<P>(y.cass, (double)dcass, dt);
  fe<P>(y.cansr, (double)dcansr, dt);
  fe<P>(y.cajsr, (double)dcajsr, dt);
}

// One cell step on one thread: rates at (t, y); if `update`, the
// Rush-Larsen / forward-Euler update of y by dt. `cur` receives the
// currents at (t, y).
template <class P, bool kCipa = false>
__device__ __forceinline__ void step(Y<typename P::G> &y, const Par<typename P::G> &q, double t, double dt,
                                     int stim_mode, bool update, Cur<typename P::G> &cur) {
  using G = typename P::G;
  const Ctx<G> c = context<P>(y, q, t, stim_mode);
  Part<G> p[4], s;
#pragma unroll
  for (int k = 0; k < kNumSums; ++k) s.f[k] = (G)0;
  role<P, kCipa, 0>(y, q, c, dt, update, p[0]);
  role<P, kCipa, 1>(y, q, c, dt, update, p[1]);
  role<P, kCipa, 2>(y, q, c, dt, update, p[2]);
  role<P, kCipa, 3>(y, q, c, dt, update, p[3]);
  add_part<kIK1InNa<P>>(s, p[0], 0);
  add_part<kIK1InNa<P>>(s, p[1], 1);
  add_part<kIK1InNa<P>>(s, p[2], 2);
  add_part<kIK1InNa<P>>(s, p[3], 3);
  combine<P>(y, q, s, dt, update, cur);
}
// Store only the states a role owns (the warp-specialised kernel: each warp
// holds stale copies of the other roles' gates). Role 0 also owns the FP64
// states every role carries (V, CaMKt, ions); xk1 belongs to the group that
// evaluates IK1 (kIK1Na: the Na group).
template <bool kCipa, bool kIK1Na, class G>
__device__ __forceinline__ void store_role(int role, const Y<G> &y, double *__restrict__ s, int64_t ld, int64_t i) {
#define CEP_ST_ORD(n) s[n * ld + i] = y.n;
#define CEP_ST_CIPA(n) s[cipa::n * ld + i] = y.n;
  if (role == (kIK1Na ? 0 : 1)) {
    if constexpr (kCipa)
      CEP_ST_CIPA(xk1)
    else
      CEP_ST_ORD(xk1)
  }
  if constexpr (!kCipa) {
    if (role == 0) {
      CEP_ST_ORD(V) CEP_ST_ORD(CaMKt) CEP_ST_ORD(cass) CEP_ST_ORD(nai) CEP_ST_ORD(nass) CEP_ST_ORD(ki)
      CEP_ST_ORD(kss) CEP_ST_ORD(cansr) CEP_ST_ORD(cajsr) CEP_ST_ORD(cai)
      CEP_ST_ORD(m) CEP_ST_ORD(hf) CEP_ST_ORD(hs) CEP_ST_ORD(j) CEP_ST_ORD(hsp) CEP_ST_ORD(jp) CEP_ST_ORD(mL)
      CEP_ST_ORD(hL) CEP_ST_ORD(hLp)
    } else if (role == 1) {
      CEP_ST_ORD(a) CEP_ST_ORD(iF) CEP_ST_ORD(iS) CEP_ST_ORD(ap) CEP_ST_ORD(iFp) CEP_ST_ORD(iSp)
      CEP_ST_ORD(xs1) CEP_ST_ORD(xs2) CEP_ST_ORD(xrf) CEP_ST_ORD(xrs)
    } else if (role == 2) {
      CEP_ST_ORD(d) CEP_ST_ORD(ff) CEP_ST_ORD(fs) CEP_ST_ORD(fcaf) CEP_ST_ORD(fcas) CEP_ST_ORD(jca)
      CEP_ST_ORD(ffp) CEP_ST_ORD(fcafp) CEP_ST_ORD(nca) CEP_ST_ORD(Jrelnp) CEP_ST_ORD(Jrelp)
    }
  } else {
    if (role == 0) {
      CEP_ST_CIPA(V) CEP_ST_CIPA(CaMKt) CEP_ST_CIPA(cass) CEP_ST_CIPA(nai) CEP_ST_CIPA(nass) CEP_ST_CIPA(ki)
      CEP_ST_CIPA(kss) CEP_ST_CIPA(cansr) CEP_ST_CIPA(cajsr) CEP_ST_CIPA(cai)
      CEP_ST_CIPA(m) CEP_ST_CIPA(hf) CEP_ST_CIPA(hs) CEP_ST_CIPA(j) CEP_ST_CIPA(hsp) CEP_ST_CIPA(jp)
      CEP_ST_CIPA(mL) CEP_ST_CIPA(hL) CEP_ST_CIPA(hLp)
    } else if (role == 1) {
      CEP_ST_CIPA(a) CEP_ST_CIPA(iF) CEP_ST_CIPA(iS) CEP_ST_CIPA(ap) CEP_ST_CIPA(iFp) CEP_ST_CIPA(iSp)
      CEP_ST_CIPA(xs1) CEP_ST_CIPA(xs2)
    } else if (role == 2) {
      CEP_ST_CIPA(d) CEP_ST_CIPA(ff) CEP_ST_CIPA(fs) CEP_ST_CIPA(fcaf) CEP_ST_CIPA(fcas) CEP_ST_CIPA(jca)
      CEP_ST_CIPA(ffp) CEP_ST_CIPA(fcafp) CEP_ST_CIPA(nca) CEP_ST_CIPA(Jrelnp) CEP_ST_CIPA(Jrelp)
    } else {
      CEP_ST_CIPA(IC1) CEP_ST_CIPA(IC2) CEP_ST_CIPA(C1) CEP_ST_CIPA(C2) CEP_ST_CIPA(O) CEP_ST_CIPA(IO)
      CEP_ST_CIPA(IObound) CEP_ST_CIPA(Obound) CEP_ST_CIPA(Cbound)
    }
  }
#undef CEP_ST_ORD
#undef CEP_ST_CIPA
}

// Hill factor of ___applyDrugEffect (Ohara_Rudy_2011.cpp:469-485): block only
// when both IC50 and h exceed 10E-14 (the reference reads NA as 0).
__device__ __forceinline__ double hill_factor(double conc, double ic50, double h) {
  return (ic50 > 10E-14 && h > 10E-14) ? 1. / (1. + ::pow(conc / ic50, h)) : 1.;
}

// initConsts(celltype, conc, ic50, is_dutta) for one instance
// (Ohara_Rudy_2011.cpp:494-678 and :722-738), written into the parameter
// block, and the model's initial STATES. `quirks` reproduces the reference's
// documented quirks (celltype forced to endo, the mis-indexed Dutta scaling,
// the drug block of PCa not reaching the derived permeabilities, and the
// STATES enum value d = 25 used as the fcafp step). `neo` is the
// CEPCell_NEO build of the model (CEPCell_NEO/cellmodels/Ohara_Rudy_2011.cpp:
// 456-520): celltype honoured, ___applyDutta on the intended constants and
// the Hill block both applied after ___initConsts has derived PCap, PCaNa
// and PCaK from PCa, which therefore stay unscaled; fcafp steps normally.
__device__ __forceinline__ void init_instance(double *__restrict__ par, double *__restrict__ s, int64_t ld,
                                              int64_t i, double celltype_in, double conc,
                                              const double *__restrict__ hill, bool dutta, bool quirks,
                                              bool neo = false) {
  if (neo) quirks = false;
  const double ct = quirks ? 0.0 : celltype_in;
  double GNaL = ct == 1.0 ? 0.0075 * 0.6 : 0.0075;
  double Gto = ct == 1.0 ? 0.02 * 4.0 : ct == 2.0 ? 0.02 * 4.0 : 0.02;
  double PCa = ct == 1.0 ? 0.0001 * 1.2 : ct == 2.0 ? 0.0001 * 2.5 : 0.0001;
  double GKr = ct == 1.0 ? 0.046 * 1.3 : ct == 2.0 ? 0.046 * 0.8 : 0.046;
  double GKs = ct == 1.0 ? 0.0034 * 1.4 : 0.0034;
  double GK1 = ct == 1.0 ? 0.1908 * 1.2 : ct == 2.0 ? 0.1908 * 1.3 : 0.1908;
  double GKb = ct == 1.0 ? 0.003 * 0.6 : 0.003;
  double Gncx = ct == 1.0 ? 0.0008 * 1.1 : ct == 2.0 ? 0.0008 * 1.4 : 0.0008;
  double Pnak = ct == 1.0 ? 30 * 0.9 : ct == 2.0 ? 30 * 0.7 : 30;
  double cmdnmax = ct == 1.0 ? 0.05 * 1.3 : 0.05;
  double upScale = ct == 1.0 ? 1.3 : 1.0;
  double Aff = 0.6, tjca = 75.0, H = 1e-7, GNa = 75;
  const double Afs = 1.0 - Aff;  // derived before the Dutta quirk scales Aff
  double PCap = 1.1 * PCa, PCaNa = 0.00125 * PCa, PCaK = 0.0003574 * PCa;
  double PCaNap = 0.00125 * PCap, PCaKp = 0.0003574 * PCap;
  if (dutta) {
    if (quirks) {  // ___applyDutta as written (Ohara_Rudy_2011.cpp:460-467)
      Aff *= 1.870; GNaL *= 1.013; tjca *= 1.698; H *= 1.007;
    } else {
      GKs *= 1.870; GKr *= 1.013; GK1 *= 1.698; PCa *= 1.007; GNaL *= 2.661;
      if (!neo) {
        PCap = 1.1 * PCa; PCaNa = 0.00125 * PCa; PCaK = 0.0003574 * PCa;
        PCaNap = 0.00125 * PCap; PCaKp = 0.0003574 * PCap;
      }
    }
  }
  if (hill) {
    PCa *= hill_factor(conc, hill[0], hill[1]);
    GK1 *= hill_factor(conc, hill[2], hill[3]);
    GKs *= hill_factor(conc, hill[4], hill[5]);
    GNa *= hill_factor(conc, hill[6], hill[7]);
    GNaL *= hill_factor(conc, hill[8], hill[9]);
    Gto *= hill_factor(conc, hill[10], hill[11]);
    GKr *= hill_factor(conc, hill[12], hill[13]);
    if (!quirks && !neo) {
      PCap = 1.1 * PCa; PCaNa = 0.00125 * PCa; PCaK = 0.0003574 * PCa;
      PCaNap = 0.00125 * PCap; PCaKp = 0.0003574 * PCap;
    }
  }
  double *p = par + i;
  p[P_GNa * ld] = GNa; p[P_GNaL * ld] = GNaL; p[P_Gto * ld] = Gto; p[P_PCa * ld] = PCa;
  p[P_PCap * ld] = PCap; p[P_PCaNa * ld] = PCaNa; p[P_PCaK * ld] = PCaK; p[P_PCaNap * ld] = PCaNap;
  p[P_PCaKp * ld] = PCaKp; p[P_GKr * ld] = GKr; p[P_GKs * ld] = GKs; p[P_GK1 * ld] = GK1;
  p[P_GKb * ld] = GKb; p[P_Gncx * ld] = Gncx; p[P_Pnak * ld] = Pnak; p[P_cmdnmax * ld] = cmdnmax;
  p[P_upScale * ld] = upScale; p[P_Aff * ld] = Aff; p[P_Afs * ld] = Afs; p[P_tjca * ld] = tjca;
  p[P_H * ld] = H; p[P_celltype * ld] = ct; p[P_fcafp_dt * ld] = quirks ? 25.0 : 0.0;
  p[P_amp * ld] = -80; p[P_BCL * ld] = 1000.0; p[P_stim_start * ld] = 10.0; p[P_duration * ld] = 0.5;
  // initial STATES (Ohara_Rudy_2011.cpp:494-678)
  const double y0[kNumStates] = {-87, 0, 1e-4, 7, 7, 145, 145, 1.2, 1.2, 1e-4, 0, 1, 1, 1, 1, 1, 0, 1, 1, 0, 1,
                                 1, 0, 1, 1, 0, 1, 1, 1, 1, 1, 1, 1, 0, 0, 0, 0, 0, 1, 0, 0};
#pragma unroll
  for (int k2 = 0; k2 < kNumStates; ++k2) s[k2 * ld + i] = y0[k2];
}

// initConsts(type, conc, hill) of CiPA-ORd v1 2017 for one instance
// (ohara_rudy_cipa_v1_2017.cpp:1246-1501 active block and :1515-1539): the
// Hill block of seven channels and the dynamic-hERG drug parameters
// hill[14..18] = Kmax, Ku, n, halfmax, Vhalf (zero keeps the model value);
// hill[19] = Kt, the trapping rate the reference leaves at 0. The binding
// rate Kmax*Ku*D^n/(D^n + halfmax) is constant per instance (D is) and is
// folded here. `quirks` forces endo and leaves the derived permeabilities
// unblocked, as the reference does.
__device__ __forceinline__ void init_instance_cipa(double *__restrict__ par, double *__restrict__ s, int64_t ld,
                                                   int64_t i, double celltype_in, double conc,
                                                   const double *__restrict__ hill, bool quirks) {
  const double ct = quirks ? 0.0 : celltype_in;
  const double GNaL_b = 0.019957499999999975, PCa_b = 0.0001007, GKr_b = 0.04658545454545456;
  const double GKs_b = 0.006358000000000001, GK1_b = 0.3239783999999998;
  double GNaL = ct == 1.0 ? GNaL_b * 0.6 : GNaL_b;
  double Gto = ct == 1.0 ? 0.02 * 4.0 : ct == 2.0 ? 0.02 * 4.0 : 0.02;
  double PCa = ct == 1.0 ? PCa_b * 1.2 : ct == 2.0 ? PCa_b * 2.5 : PCa_b;
  double GKr = ct == 1.0 ? GKr_b * 1.3 : ct == 2.0 ? GKr_b * 0.8 : GKr_b;
  double GKs = ct == 1.0 ? GKs_b * 1.4 : GKs_b;
  double GK1 = ct == 1.0 ? GK1_b * 1.2 : ct == 2.0 ? GK1_b * 1.3 : GK1_b;
  const double GKb = ct == 1.0 ? 0.003 * 0.6 : 0.003;
  const double Gncx = ct == 1.0 ? 0.0008 * 1.1 : ct == 2.0 ? 0.0008 * 1.4 : 0.0008;
  const double Pnak = ct == 1.0 ? 30 * 0.9 : ct == 2.0 ? 30 * 0.7 : 30;
  const double cmdnmax = ct == 1.0 ? 0.05 * 1.3 : 0.05;
  const double upScale = ct == 1.0 ? 1.3 : 1.0;
  double GNa = 75;
  double PCap = 1.1 * PCa, PCaNa = 0.00125 * PCa, PCaK = 0.0003574 * PCa;
  double PCaNap = 0.00125 * PCap, PCaKp = 0.0003574 * PCap;
  double Kmax = 0, Ku = 0, nn = 1, halfmax = 1, Vhalf = 1, Kt = 0;
  if (hill) {
    PCa *= hill_factor(conc, hill[0], hill[1]);
    GK1 *= hill_factor(conc, hill[2], hill[3]);
    GKs *= hill_factor(conc, hill[4], hill[5]);
    GNa *= hill_factor(conc, hill[6], hill[7]);
    GNaL *= hill_factor(conc, hill[8], hill[9]);
    Gto *= hill_factor(conc, hill[10], hill[11]);
    GKr *= hill_factor(conc, hill[12], hill[13]);
    if (!quirks) {
      PCap = 1.1 * PCa; PCaNa = 0.00125 * PCa; PCaK = 0.0003574 * PCa;
      PCaNap = 0.00125 * PCap; PCaKp = 0.0003574 * PCap;
    }
    if (hill[14] > 10E-14) Kmax = hill[14];
    if (hill[15] > 10E-14) Ku = hill[15];
    if (hill[16] > 10E-14) nn = hill[16];
    if (hill[17] > 10E-14) halfmax = hill[17];
    // quirk: the reference's `> 10E-14` guard drops every negative Vhalf
    if (quirks ? hill[18] > 10E-14 : hill[18] != 0.0) Vhalf = hill[18];
    if (hill[19] > 10E-14) Kt = hill[19];
  }
  const double Dn = ::exp(nn * ::log(conc));
  const double bind = (Kmax * Ku * Dn) / (Dn + halfmax);
  double *p = par + i;
  p[P_GNa * ld] = GNa; p[P_GNaL * ld] = GNaL; p[P_Gto * ld] = Gto; p[P_PCa * ld] = PCa;
  p[P_PCap * ld] = PCap; p[P_PCaNa * ld] = PCaNa; p[P_PCaK * ld] = PCaK; p[P_PCaNap * ld] = PCaNap;
  p[P_PCaKp * ld] = PCaKp; p[P_GKr * ld] = GKr; p[P_GKs * ld] = GKs; p[P_GK1 * ld] = GK1;
  p[P_GKb * ld] = GKb; p[P_Gncx * ld] = Gncx; p[P_Pnak * ld] = Pnak; p[P_cmdnmax * ld] = cmdnmax;
  p[P_upScale * ld] = upScale; p[P_Aff * ld] = 0.6; p[P_Afs * ld] = 1.0 - 0.6; p[P_tjca * ld] = 75.0;
  p[P_H * ld] = 1e-7; p[P_celltype * ld] = ct; p[P_fcafp_dt * ld] = 0.0;
  p[P_amp * ld] = -80; p[P_BCL * ld] = 1000.0; p[P_stim_start * ld] = 10.0; p[P_duration * ld] = 0.5;
  p[P_bind * ld] = bind; p[P_Ku * ld] = Ku; p[P_Kt * ld] = Kt; p[P_Vhalf * ld] = Vhalf;
  const double y0[cipa::kNumStates] = {
      -88.00190465, 0.0125840447, 8.49e-05, 7.268004498, 7.268089977, 144.6555918, 144.6555651, 1.619574538,
      1.571234014, 8.6e-05, 0.007344121102, 0.6981071913, 0.6980895801, 0.6979908432, 0.4549485525,
      0.6979245865, 0.0001882617273, 0.5008548855, 0.2693065357, 0.001001097687, 0.9995541745, 0.5865061736,
      0.0005100862934, 0.9995541823, 0.6393399482, 2.34e-9, 0.9999999909, 0.9102412777, 0.9999999909,
      0.9998046777, 0.9999738312, 0.9999999909, 0.9999999909, 0.002749414044, 0.999637, 6.83208e-05,
      1.80145e-08, 8.26619e-05, 0.00015551, 5.67623e-05, 0, 0, 0, 0, 0.2707758025, 0.0001928503426,
      0.9967597594, 2.5e-7, 3.12e-7};
#pragma unroll
  for (int k2 = 0; k2 < cipa::kNumStates; ++k2) s[k2 * ld + i] = y0[k2];
  s[cipa::D * ld + i] = conc;
}

}  // namespace ord
}  // namespace cep
