// ToR-ORd (Tomek et al. 2019), one cell per thread, templated on the
// precision policy (cep_device.cuh).
//
// Equations: CEPCell_NEO/cellmodels/Tomek_model.cpp computeRates
// (:1171-1440) with the endo/epi/mid constants of ___initEndo/Epi/Mid
// (:506-1134) and the Hill hook of initConsts(celltype, conc, hill)
// (:1149-1168). The reference's solveAnalytical is empty (it integrates
// with CVODE only); the fixed-step scheme is the ORd one: Rush-Larsen for
// every (inf - y)/tau gate, the Jrel relaxations and nca; forward Euler for
// CaMKt, the IKr Markov states, V and the concentrations.
#pragma once
#include "cep_device.cuh"

namespace cep {
namespace tomek {

constexpr int kNumStates = 43;
enum : int {
  V = 0, CaMKt, cass, nai, nass, ki, kss, cansr, cajsr, cai, m, h, j, hp, jp, mL, hL, hLp, a, iF, iS, ap, iFp, iSp,
  d, ff, fs, fcaf, fcas, jca, ffp, fcafp, nca_ss, nca_i, C1, C2, C3, I, O, xs1, xs2, Jrel_np, Jrel_p
};
// per-instance parameters (celltype- and drug-dependent), then the
// constants that need exp/log (evaluated once at init), then pacing
enum : int {
  P_GNa = 0, P_GNaL, P_Gto, P_PCa, P_PCap, P_PCaNa, P_PCaK, P_PCaNap, P_PCaKp, P_GKr, P_GKs, P_GK1, P_GKb,
  P_Gncx, P_Pnak, P_cmdnmax, P_upScale, P_epi, P_jrel_scale, P_gamma_cao, P_gamma_nao, P_gamma_ko, P_ECl, P_constA,
  P_amp, P_BCL, P_stim_start, P_duration, kNumParams
};

namespace k {
constexpr double nao = 140.0, cao = 1.8, ko = 5.0, clo = 150.0, R = 8314, T = 310, F = 96485, L = 0.01, rad = 0.0011;
constexpr double KmCaMK = 0.15, aCaMK = 0.05, bCaMK = 0.00068, CaMKo = 0.05, KmCaM = 0.0015;
constexpr double kmcmdn = 0.00238, trpnmax = 0.07, kmtrpn = 0.0005, BSRmax = 0.047, KmBSR = 0.00087;
constexpr double BSLmax = 1.124, KmBSL = 0.0087, csqnmax = 10, kmcsqn = 0.8, cli = 24.0, PKNa = 0.01833;
constexpr double thL = 200, thLp = 3.0 * thL, Kmn = 0.002, k2n = 500, Aff = 0.6, Afs = 1.0 - Aff, tjca = 75;
constexpr double dielConstant = 74, fracSS = 0.8, alpha_1 = 0.154375, beta_1 = 0.1911, ncxSS = 0.35;
constexpr double kna1 = 15, kna2 = 5, kna3 = 88.12, kasymm = 12.5, wna = 6e4, wca = 6e4, wnaca = 5e3;
constexpr double kcaon = 1.5e6, kcaoff = 5e3, qna = 0.5224, qca = 0.167, KmCaAct = 150e-6;
constexpr double k1p = 949.5, k1m = 182.4, k2p = 687.2, k2m = 39.4, k3p = 1899, k3m = 79300, k4p = 639, k4m = 40;
constexpr double Knai0 = 9.073, Knao0 = 27.78, delta = -0.155, Kki = 0.5, Kko = 0.3582, MgADP = 0.05, MgATP = 9.8;
constexpr double Kmgatp = 1.698e-7, H = 1e-7, eP = 4.2, Khp = 1.698e-7, Knap = 224, Kxkur = 292;
constexpr double PNab = 1.9239e-09, PCab = 5.9194e-08, GpCa = 5e-04, KmCap = 0.0005, GClCa = 0.2843;
constexpr double GClb = 1.98e-3, KdClCa = 0.1, tauNa = 2.0, tauK = 2.0, tauCa = 0.2, bt = 4.75, btp = 1.25 * bt;
constexpr double a_rel = 0.5 * bt, a_relp = 0.5 * btp, cajsr_half = 1.7, Jrel_b = 1.5378, Jup_b = 1.0;
constexpr double vcell = 1000.0 * 3.14 * rad * rad * L, Ageo = 2.0 * 3.14 * rad * rad + 2.0 * 3.14 * rad * L;
constexpr double Acap = 2.0 * Ageo, vmyo = 0.68 * vcell, vnsr = 0.0552 * vcell, vjsr = 0.0048 * vcell;
constexpr double vss = 0.02 * vcell;
constexpr double h10 = kasymm + 1.0 + (nao / kna1) * (1.0 + nao / kna2), h11 = (nao * nao) / (h10 * kna1 * kna2);
constexpr double k1n = (1.0 / h10) * cao * kcaon, k2n_ = kcaoff, k5n = kcaoff;  // NaCa (same in i and ss)
constexpr double b1 = k1m * MgADP, a2 = k2p, a4 = ((k4p * MgATP) / Kmgatp) / (1.0 + MgATP / Kmgatp);
constexpr double FRT = F / (R * T), RTF = (R * T) / F, Io = (0.5 * (nao + ko + clo + 4.0 * cao)) / 1000.0;
constexpr double sqrt_ko5 = 1.0;  // sqrt(ko / 5)
constexpr double Kmgatp_fac = 1.0 + MgATP / Kmgatp;
// Acap / (F V) scalings of the concentration equations
constexpr double c_myo = Acap / (F * vmyo), c_ss = Acap / (F * vss);
}  // namespace k

template <class G>
struct Y {
  double V, CaMKt, cass, nai, nass, ki, kss, cansr, cajsr, cai, m, h, j, hp, jp, mL, hL, hLp, a, iF, iS, ap, iFp, iSp,
      d, ff, fs, fcaf, fcas, jca, ffp, fcafp, nca_ss, nca_i, C1, C2, C3, I, O, xs1, xs2, Jrel_np, Jrel_p;
};
template <class G>
struct Par {
  G GNa, GNaL, Gto, PCa, PCap, PCaNa, PCaK, PCaNap, PCaKp, GKr, GKs, GK1, GKb, Gncx, Pnak, cmdnmax, upScale;
  G epi, jrel_scale, gamma_cao, gamma_nao, gamma_ko, ECl, constA;
  double amp, BCL, stim_start, duration;
};
template <class G>
struct Cur {
  G INa, INaL, Ito, ICaL, IKr, IKs, IK1, dVdt;
};

#define CEP_TOMEK_FIELDS(X) X(V) X(CaMKt) X(cass) X(nai) X(nass) X(ki) X(kss) X(cansr) X(cajsr) X(cai) X(m) X(h) \
  X(j) X(hp) X(jp) X(mL) X(hL) X(hLp) X(a) X(iF) X(iS) X(ap) X(iFp) X(iSp) X(d) X(ff) X(fs) X(fcaf) X(fcas) X(jca) \
  X(ffp) X(fcafp) X(nca_ss) X(nca_i) X(C1) X(C2) X(C3) X(I) X(O) X(xs1) X(xs2) X(Jrel_np) X(Jrel_p)

template <class G>
__device__ __forceinline__ void load(Y<G> &y, const double *__restrict__ s_, int64_t ld, int64_t i) {
#define CEP_LD(n) y.n = s_[n * ld + i];
  CEP_TOMEK_FIELDS(CEP_LD)
#undef CEP_LD
}
template <class G>
__device__ __forceinline__ void store(const Y<G> &y, double *__restrict__ s_, int64_t ld, int64_t i) {
#define CEP_ST(n) s_[n * ld + i] = y.n;
  CEP_TOMEK_FIELDS(CEP_ST)
#undef CEP_ST
}
template <class G>
__device__ __forceinline__ void load_par(Par<G> &q, const double *__restrict__ p, int64_t ld, int64_t i) {
#define CEP_LP(n) q.n = (G)p[P_##n * ld + i];
  CEP_LP(GNa) CEP_LP(GNaL) CEP_LP(Gto) CEP_LP(PCa) CEP_LP(PCap) CEP_LP(PCaNa) CEP_LP(PCaK) CEP_LP(PCaNap)
  CEP_LP(PCaKp) CEP_LP(GKr) CEP_LP(GKs) CEP_LP(GK1) CEP_LP(GKb) CEP_LP(Gncx) CEP_LP(Pnak) CEP_LP(cmdnmax)
  CEP_LP(upScale) CEP_LP(epi) CEP_LP(jrel_scale) CEP_LP(gamma_cao) CEP_LP(gamma_nao) CEP_LP(gamma_ko) CEP_LP(ECl) CEP_LP(constA)
#undef CEP_LP
  q.amp = p[P_amp * ld + i]; q.BCL = p[P_BCL * ld + i]; q.stim_start = p[P_stim_start * ld + i];
  q.duration = p[P_duration * ld + i];
}

// vffrt / (e^{z vfrt} - 1) and e^{z vfrt}; the mixed form evaluates the
// ratio through x/(e^x - 1), finite at V = 0
template <class P, int z>
__device__ __forceinline__ void ghk(double V, typename P::G v, typename P::G &fac, typename P::G &e) {
  using G = typename P::G;
  if constexpr (P::kMixed) {
    const G x = (G)z * v * (G)k::FRT;
    e = P::ex(x);
    fac = ghk_factor(x) * (G)(k::F / z);
  } else {
    const double vffrt = (V * k::F * k::F) / (k::R * k::T);
    const double ee = exp_f64((double)z * ((V * k::F) / (k::R * k::T)));
    e = ee;
    fac = div64(vffrt, ee - 1.0);
  }
}

// Debye-Hueckel activity coefficient exp(-A z^2 (sqrt(I)/(1+sqrt(I)) - 0.3 I))
template <class P>
__device__ __forceinline__ typename P::G activity(typename P::G constA_z2, typename P::G ionic) {
  using G = typename P::G;
  const G s = P::sq(ionic);
  return P::ex(-constA_z2 * (P::dv(s, (G)1 + s) - (G)0.3 * ionic));
}

// Sodium-calcium exchanger cycle for one compartment (i or ss): the two
// fluxes JncxNa, JncxCa of the reference's four-state scheme.
template <class P>
__device__ __forceinline__ void naca(typename P::G na, typename P::G ca, typename P::G hna, typename P::G hca,
                                     typename P::G &JNa, typename P::G &JCa) {
  using G = typename P::G;
  const G one = (G)1;
  const G h7 = one + (G)(k::nao / k::kna3) * (one + P::rc(hna));
  const G h8 = P::dv((G)k::nao, (G)k::kna3 * hna * h7);
  const G k3pp = h8 * (G)k::wnaca;
  const G h1 = one + na * (G)(1.0 / k::kna3) * (one + hna);
  const G h2 = P::dv(na * hna, (G)k::kna3 * h1);
  const G k4pp = h2 * (G)k::wnaca;
  const G h4 = one + na * (G)(1.0 / k::kna1) * (one + na * (G)(1.0 / k::kna2));
  const G h5 = P::dv(na * na, h4 * (G)(k::kna1 * k::kna2));
  const G k7 = h5 * h2 * (G)k::wna;
  const G k8 = h8 * (G)(k::h11 * k::wna);
  const G k3 = P::rc(h7) * (G)k::wca + k3pp;
  const G k4 = P::dv(P::rc(h1) * (G)k::wca, hca) + k4pp;
  const G k6 = P::rc(h4) * ca * (G)k::kcaon;
  const G k1 = (G)k::k1n, k2 = (G)k::k2n_, k5 = (G)k::k5n;
  const G x1 = k2 * k4 * (k7 + k6) + k5 * k7 * (k2 + k3);
  const G x2 = k1 * k7 * (k4 + k5) + k4 * k6 * (k1 + k8);
  const G x3 = k1 * k3 * (k7 + k6) + k8 * k6 * (k2 + k3);
  const G x4 = k2 * k8 * (k4 + k5) + k3 * k5 * (k1 + k8);
  const G inv = P::rc(x1 + x2 + x3 + x4);
  const G E1 = x1 * inv, E2 = x2 * inv, E3 = x3 * inv, E4 = x4 * inv;
  JNa = ((G)3 * (E4 * k7 - E1 * k8) + E3 * k4pp) - E2 * k3pp;
  JCa = E2 * k2 - E1 * k1;
}

template <class P>
__device__ __forceinline__ void step(Y<typename P::G> &y, const Par<typename P::G> &q, double t, double dt,
                                     int stim_mode, bool update, Cur<typename P::G> &cur) {
  using G = typename P::G;
  const G v = (G)y.V, one = (G)1;
  bool on;
  if (stim_mode < 0) {
    on = t >= q.stim_start && (t - q.stim_start) - floor((t - q.stim_start) / q.BCL) * q.BCL <= q.duration;
  } else {
    on = stim_mode != 0;
  }
  const G Istim = on ? (G)q.amp : (G)0;
  const G cass_ = (G)y.cass, cai_ = (G)y.cai, nai_ = (G)y.nai, nass_ = (G)y.nass, ki_ = (G)y.ki, kss_ = (G)y.kss;
  const G cajsr_ = (G)y.cajsr, cansr_ = (G)y.cansr;
  // gates
  const G hLss = P::rc(one + P::ex((v + (G)87.61) * (G)(1.0 / 7.488)));
  const G hLssp = P::rc(one + P::ex((v + (G)93.81) * (G)(1.0 / 7.488)));
  const G jcass = P::rc(one + P::ex((v + (G)18.08) * (G)(1.0 / 2.7916)));
  const G mss = P::rc(p2(one + P::ex(-(v + (G)56.86) * (G)(1.0 / 9.03))));
  const G tm = (G)0.1292 * P::ex(-p2((v + (G)45.79) * (G)(1.0 / 15.54))) + (G)0.06487 * P::ex(-p2((v - (G)4.823) * (G)(1.0 / 51.12)));
  const G mLss = P::rc(one + P::ex(-(v + (G)42.85) * (G)(1.0 / 5.264)));
  const G ass = P::rc(one + P::ex(-(v - (G)14.34) * (G)(1.0 / 14.82)));
  const G ta = P::dv((G)1.0515, P::rc((G)1.2089 * (one + P::ex(-(v - (G)18.4099) * (G)(1.0 / 29.3814)))) +
                                     P::dv((G)3.5, one + P::ex((v + (G)100.0) * (G)(1.0 / 29.3814))));
  const G dss = v >= (G)31.4978 ? one : (G)1.0763 * P::ex((G)-1.007 * P::ex((G)-0.0829 * v));
  const G td = (G)0.6 + P::rc(P::ex((G)-0.05 * (v + (G)6.0)) + P::ex((G)0.09 * (v + (G)14.0)));
  const G fss = P::rc(one + P::ex((v + (G)19.58) * (G)(1.0 / 3.696)));
  const G tff = (G)7.0 + P::rc((G)0.0045 * P::ex(-(v + (G)20.0) * (G)0.1) + (G)0.0045 * P::ex((v + (G)20.0) * (G)0.1));
  const G tfs = (G)1000.0 + P::rc((G)3.5e-05 * P::ex(-(v + (G)5.0) * (G)0.25) + (G)3.5e-05 * P::ex((v + (G)5.0) * (G)(1.0 / 6.0)));
  const G km2n = (G)y.jca;
  const G anca_ss = P::rc(P::dv((G)k::k2n, km2n) + p4(one + P::dv((G)k::Kmn, cass_)));
  const G anca_i = P::rc(P::dv((G)k::k2n, km2n) + p4(one + P::dv((G)k::Kmn, cai_)));
  const G xs1ss = P::rc(one + P::ex(-(v + (G)11.6) * (G)(1.0 / 8.932)));
  const G txs1 = (G)817.3 + P::rc((G)0.0002326 * P::ex((v + (G)48.28) * (G)(1.0 / 17.8)) + (G)0.001292 * P::ex(-(v + (G)210.0) * (G)(1.0 / 230.0)));
  const G assp = P::rc(one + P::ex(-(v - (G)24.34) * (G)(1.0 / 14.82)));
  const G tfcaf = (G)7.0 + P::rc((G)0.04 * P::ex(-(v - (G)4.0) * (G)(1.0 / 7.0)) + (G)0.04 * P::ex((v - (G)4.0) * (G)(1.0 / 7.0)));
  const G tfcas = (G)100.0 + P::rc((G)0.00012 * P::ex(-v * (G)(1.0 / 3.0)) + (G)0.00012 * P::ex(v * (G)(1.0 / 7.0)));
  const G txs2 = P::rc((G)0.01 * P::ex((v - (G)50.0) * (G)0.05) + (G)0.0193 * P::ex(-(v + (G)66.54) * (G)(1.0 / 31.0)));
  const G CaMKb = P::dv((G)k::CaMKo * (one - (G)y.CaMKt), one + P::dv((G)k::KmCaM, cass_));
  const G hss = P::rc(p2(one + P::ex((v + (G)71.55) * (G)(1.0 / 7.43))));
  const bool hi = v >= (G)-40.0;
  const G ah = hi ? (G)0 : (G)0.057 * P::ex(-(v + (G)80.0) * (G)(1.0 / 6.8));
  const G bh = hi ? P::dv((G)0.77, (G)0.13 * (one + P::ex(-(v + (G)10.66) * (G)(1.0 / 11.1))))
                  : (G)2.7 * P::ex((G)0.079 * v) + (G)310000.0 * P::ex((G)0.3485 * v);
  const G th = P::rc(ah + bh);
  const G aj = hi ? (G)0
                  : P::dv(((G)-25428.0 * P::ex((G)0.2444 * v) - (G)6.948e-06 * P::ex((G)-0.04391 * v)) * (v + (G)37.78),
                          one + P::ex((G)0.311 * (v + (G)79.23)));
  const G bj = hi ? P::dv((G)0.6 * P::ex((G)0.057 * v), one + P::ex((G)-0.1 * (v + (G)32.0)))
                  : P::dv((G)0.02424 * P::ex((G)-0.01052 * v), one + P::ex((G)-0.1378 * (v + (G)40.14)));
  const G tj = P::rc(aj + bj);
  const G hssp = P::rc(p2(one + P::ex((v + (G)77.55) * (G)(1.0 / 7.43))));
  const G iss = P::rc(one + P::ex((v + (G)43.94) * (G)(1.0 / 5.711)));
  const G delta_epi = q.epi != (G)0 ? one - P::dv((G)0.95, one + P::ex((v + (G)70.0) * (G)0.2)) : one;
  const G tiF = ((G)4.562 + P::rc((G)0.3933 * P::ex(-(v + (G)100.0) * (G)0.01) + (G)0.08004 * P::ex((v + (G)50.0) * (G)(1.0 / 16.59)))) * delta_epi;
  const G tiS = ((G)23.62 + P::rc((G)0.001416 * P::ex(-(v + (G)96.52) * (G)(1.0 / 59.05)) + (G)1.78e-08 * P::ex((v + (G)114.1) * (G)(1.0 / 8.079)))) * delta_epi;
  const G dti_develop = (G)1.354 + P::dv((G)0.0001, P::ex((v - (G)167.4) * (G)(1.0 / 15.89)) + P::ex(-(v - (G)12.23) * (G)(1.0 / 0.2154)));
  const G dti_recover = one - P::dv((G)0.5, one + P::ex((v + (G)70.0) * (G)0.05));
  const G tiFp = dti_develop * dti_recover * tiF;
  const G tiSp = dti_develop * dti_recover * tiS;
  // IKr Markov rates
  const G vfrt = v * (G)k::FRT;
  const G alpha = (G)0.1161 * P::ex((G)0.299 * vfrt);
  const G beta = (G)0.2442 * P::ex((G)-1.604 * vfrt);
  const G alpha_2 = (G)0.0578 * P::ex((G)0.971 * vfrt);
  const G beta_2 = (G)0.000349 * P::ex((G)-1.062 * vfrt);
  const G alpha_i = (G)0.2533 * P::ex((G)0.5953 * vfrt);
  const G beta_i = (G)0.06525 * P::ex((G)-0.8209 * vfrt);
  const G alpha_C2ToI = (G)5.2e-05 * P::ex((G)1.525 * vfrt);
  const G beta_ItoC2 = P::dv(beta_2 * beta_i * alpha_C2ToI, alpha_2 * alpha_i);
  // CaMK and phosphorylated fractions
  const G CaMKa = CaMKb + (G)y.CaMKt;
  const G fP = P::rc(one + P::dv((G)k::KmCaMK, CaMKa));  // fICaLp = fItop = fINap = fINaLp = fJrelp = fJupp
  // L-type channel gating
  const G f = (G)k::Aff * (G)y.ff + (G)k::Afs * (G)y.fs;
  const G Afcaf = (G)0.3 + P::dv((G)0.6, one + P::ex((v - (G)10.0) * (G)0.1));
  const G Afcas = one - Afcaf;
  const G fca = Afcaf * (G)y.fcaf + Afcas * (G)y.fcas;
  const G fp = (G)k::Aff * (G)y.ffp + (G)k::Afs * (G)y.fs;
  const G fcap = Afcaf * (G)y.fcafp + Afcas * (G)y.fcas;
  const G jca_ = (G)y.jca, d_ = (G)y.d, nss = (G)y.nca_ss, nci = (G)y.nca_i;
  const G gate_ss = (one - fP) * d_ * (f * (one - nss) + jca_ * fca * nss);
  const G gatep_ss = fP * d_ * (fp * (one - nss) + jca_ * fcap * nss);
  const G gate_i = (one - fP) * d_ * (f * (one - nci) + jca_ * fca * nci);
  const G gatep_i = fP * d_ * (fp * (one - nci) + jca_ * fcap * nci);
  // ionic strengths and activities
  const G constA = q.constA;
  const G Iss = (G)0.5 * (nass_ + kss_ + (G)k::cli + (G)4.0 * cass_) * (G)0.001;
  const G Ii = (G)0.5 * (nai_ + ki_ + (G)k::cli + (G)4.0 * cai_) * (G)0.001;
  const G g1ss = activity<P>(constA, Iss), g1i = activity<P>(constA, Ii);
  const G g4ss = activity<P>((G)4 * constA, Iss), g4i = activity<P>((G)4 * constA, Ii);
  G fac1, e1, fac2, e2;
  ghk<P, 1>(y.V, v, fac1, e1);
  ghk<P, 2>(y.V, v, fac2, e2);
  const G PhiCaL_ss = (G)4 * fac2 * (g4ss * cass_ * e2 - q.gamma_cao * (G)k::cao);
  const G PhiCaL_i = (G)4 * fac2 * (g4i * cai_ * e2 - q.gamma_cao * (G)k::cao);
  const G PhiCaK_ss = fac1 * (g1ss * kss_ * e1 - q.gamma_ko * (G)k::ko);
  const G PhiCaK_i = fac1 * (g1i * ki_ * e1 - q.gamma_ko * (G)k::ko);
  const G PhiCaNa_ss = fac1 * (g1ss * nass_ * e1 - q.gamma_nao * (G)k::nao);
  const G PhiCaNa_i = fac1 * (g1i * nai_ * e1 - q.gamma_nao * (G)k::nao);
  const G ICaL_ss = (G)k::fracSS * (q.PCa * PhiCaL_ss * gate_ss + q.PCap * PhiCaL_ss * gatep_ss);
  const G ICaL_i = (G)(1.0 - k::fracSS) * (q.PCa * PhiCaL_i * gate_i + q.PCap * PhiCaL_i * gatep_i);
  const G ICaK_ss = (G)k::fracSS * (q.PCaK * PhiCaK_ss * gate_ss + q.PCaKp * PhiCaK_ss * gatep_ss);
  const G ICaK_i = (G)(1.0 - k::fracSS) * (q.PCaK * PhiCaK_i * gate_i + q.PCaKp * PhiCaK_i * gatep_i);
  const G ICaNa_ss = (G)k::fracSS * (q.PCaNa * PhiCaNa_ss * gate_ss + q.PCaNap * PhiCaNa_ss * gatep_ss);
  const G ICaNa_i = (G)(1.0 - k::fracSS) * (q.PCaNa * PhiCaNa_i * gate_i + q.PCaNap * PhiCaNa_i * gatep_i);
  const G ICaL = ICaL_ss + ICaL_i;
  // potassium currents
  const G EK = (G)k::RTF * P::lg(P::dv((G)k::ko, ki_));
  const G vek = v - EK;
  const G AiF = P::rc(one + P::ex((v - (G)213.6) * (G)(1.0 / 151.2)));
  const G AiS = one - AiF;
  const G ii = AiF * (G)y.iF + AiS * (G)y.iS;
  const G ip = AiF * (G)y.iFp + AiS * (G)y.iSp;
  const G Ito = q.Gto * vek * ((one - fP) * (G)y.a * ii + fP * (G)y.ap * ip);
  const G IKr = q.GKr * (G)k::sqrt_ko5 * (G)y.O * vek;
  const G EKs = (G)k::RTF * P::lg(P::dv((G)(k::ko + k::PKNa * k::nao), ki_ + (G)k::PKNa * nai_));
  const G KsCa = one + P::dv((G)0.6, one + P::pw(P::dv((G)3.8e-05, cai_), (G)1.4));
  const G IKs = q.GKs * KsCa * (G)y.xs1 * (G)y.xs2 * (v - EKs);
  const G aK1 = P::dv((G)4.094, one + P::ex((G)0.1217 * (vek - (G)49.934)));
  const G bK1 = P::dv((G)15.72 * P::ex((G)0.0674 * (vek - (G)3.257)) + P::ex((G)0.0618 * (vek - (G)594.31)),
                      one + P::ex((G)-0.1629 * (vek + (G)14.207)));
  const G IK1 = q.GK1 * (G)k::sqrt_ko5 * P::dv(aK1, aK1 + bK1) * vek;
  const G xkb = P::rc(one + P::ex(-(v - (G)10.8968) * (G)(1.0 / 23.9871)));
  const G IKb = q.GKb * xkb * vek;
  // Na/K pump
  const G Knao = (G)k::Knao0 * P::ex((G)((1.0 - k::delta) / 3.0) * vfrt);
  const G Knai = (G)k::Knai0 * P::ex((G)(k::delta / 3.0) * vfrt);
  const G kok = (G)(k::ko / k::Kko);
  const G den_o = (p3(one + P::dv((G)k::nao, Knao)) + p2(one + kok)) - one;
  const G den_i = (p3(one + P::dv(nai_, Knai)) + p2(one + ki_ * (G)(1.0 / k::Kki))) - one;
  const G a3 = P::dv((G)k::k3p * p2(kok), den_o);
  const G Pp = P::dv((G)k::eP, one + (G)(k::H / k::Khp) + nai_ * (G)(1.0 / k::Knap) + ki_ * (G)(1.0 / k::Kxkur));
  const G b3 = Pp * (G)(k::k3m * k::H / k::Kmgatp_fac);
  const G a1 = P::dv((G)k::k1p * p3(P::dv(nai_, Knai)), den_i);
  const G b2 = P::dv((G)k::k2m * p3(P::dv((G)k::nao, Knao)), den_o);
  const G b4 = P::dv((G)k::k4m * p2(ki_ * (G)(1.0 / k::Kki)), den_i);
  const G B1 = (G)k::b1, A2 = (G)k::a2, A4 = (G)k::a4;
  const G x1 = A4 * a1 * A2 + b2 * b4 * b3 + A2 * b4 * b3 + b3 * a1 * A2;
  const G x2 = b2 * B1 * b4 + a1 * A2 * a3 + a3 * B1 * b4 + A2 * a3 * b4;
  const G x3 = A2 * a3 * A4 + b3 * b2 * B1 + b2 * B1 * A4 + a3 * A4 * B1;
  const G x4 = b4 * b3 * b2 + a3 * A4 * a1 + b2 * A4 * a1 + b3 * b2 * a1;
  const G inv = P::rc(x1 + x2 + x3 + x4);
  const G JnakNa = (G)3 * (x1 * inv * a3 - x2 * inv * b3);
  const G JnakK = (G)2 * (x4 * inv * B1 - x3 * inv * a1);
  const G INaK = q.Pnak * (JnakNa + JnakK);
  // sodium currents
  const G ENa = (G)k::RTF * P::lg(P::dv((G)k::nao, nai_));
  const G INa = q.GNa * (v - ENa) * p3((G)y.m) * ((one - fP) * (G)y.h * (G)y.j + fP * (G)y.hp * (G)y.jp);
  const G INaL = q.GNaL * (v - ENa) * (G)y.mL * ((one - fP) * (G)y.hL + fP * (G)y.hLp);
  const G INab = (G)k::PNab * fac1 * (nai_ * e1 - (G)k::nao);
  // Na/Ca exchangers
  const G hna = P::ex((G)k::qna * vfrt), hca = P::ex((G)k::qca * vfrt);
  G JNa_i, JCa_i, JNa_ss, JCa_ss;
  naca<P>(nai_, cai_, hna, hca, JNa_i, JCa_i);
  naca<P>(nass_, cass_, hna, hca, JNa_ss, JCa_ss);
  const G allo_i = P::rc(one + p2(P::dv((G)k::KmCaAct, cai_)));
  const G allo_ss = P::rc(one + p2(P::dv((G)k::KmCaAct, cass_)));
  const G INaCa_i = (G)(1.0 - k::ncxSS) * q.Gncx * allo_i * (JNa_i + (G)2 * JCa_i);
  const G INaCa_ss = (G)k::ncxSS * q.Gncx * allo_ss * (JNa_ss + (G)2 * JCa_ss);
  // calcium currents and chloride
  const G IpCa = P::dv((G)k::GpCa * cai_, (G)k::KmCap + cai_);
  const G ICab = (G)(4.0 * k::PCab) * fac2 * (g4i * cai_ * e2 - q.gamma_cao * (G)k::cao);
  const G IClCa = P::dv((G)k::GClCa, one + P::dv((G)k::KdClCa, cass_)) * (v - q.ECl);  // Fjunc = 1
  const G IClb = (G)k::GClb * (v - q.ECl);
  const G dV = -(INa + INaL + Ito + ICaL + (ICaNa_ss + ICaNa_i) + (ICaK_ss + ICaK_i) + IKr + IKs + IK1 + INaCa_i +
                 INaCa_ss + INaK + INab + IKb + IpCa + ICab + IClCa + IClb + Istim);
  cur.INa = INa; cur.INaL = INaL; cur.Ito = Ito; cur.ICaL = ICaL; cur.IKr = IKr; cur.IKs = IKs; cur.IK1 = IK1;
  cur.dVdt = dV;
  if (!update) return;
  // fluxes and buffers
  const G cajsr_8 = p8(P::dv((G)k::cajsr_half, cajsr_));
  const G Jrel_inf = P::dv((G)-k::a_rel * ICaL_ss, one + cajsr_8) * q.jrel_scale;
  const G Jrel_infp = P::dv((G)-k::a_relp * ICaL_ss, one + cajsr_8) * q.jrel_scale;
  const G trel = P::dv((G)k::bt, one + P::dv((G)0.0123, cajsr_));
  const G trelp = P::dv((G)k::btp, one + P::dv((G)0.0123, cajsr_));
  const G tau_rel = trel < (G)0.001 ? (G)0.001 : trel;
  const G tau_relp = trelp < (G)0.001 ? (G)0.001 : trelp;
  const G Jrel = (G)k::Jrel_b * ((one - fP) * (G)y.Jrel_np + fP * (G)y.Jrel_p);
  const G JdiffNa = (nass_ - nai_) * (G)(1.0 / k::tauNa);
  const G JdiffK = (kss_ - ki_) * (G)(1.0 / k::tauK);
  const G Jdiff = (cass_ - cai_) * (G)(1.0 / k::tauCa);
  const G Jupnp = P::dv(q.upScale * (G)0.005425 * cai_, cai_ + (G)0.00092);
  const G Jupp = P::dv(q.upScale * (G)(2.75 * 0.005425) * cai_, (cai_ + (G)0.00092) - (G)0.00017);
  const G Jleak = (G)(0.0048825 / 15.0) * cansr_;
  const G Jup = (G)k::Jup_b * (((one - fP) * Jupnp + fP * Jupp) - Jleak);
  const G Jtr = (cansr_ - cajsr_) * (G)(1.0 / 60.0);
  const G Bcass = P::rc(one + P::dv((G)(k::BSRmax * k::KmBSR), p2((G)k::KmBSR + cass_)) +
                        P::dv((G)(k::BSLmax * k::KmBSL), p2((G)k::KmBSL + cass_)));
  const G Bcai = P::rc(one + P::dv(q.cmdnmax * (G)k::kmcmdn, p2((G)k::kmcmdn + cai_)) +
                       P::dv((G)(k::trpnmax * k::kmtrpn), p2((G)k::kmtrpn + cai_)));
  const G Bcajsr = P::rc(one + P::dv((G)(k::csqnmax * k::kmcsqn), p2((G)k::kmcsqn + cajsr_)));
  const G dki = -(((Ito + IKr + IKs + IK1 + IKb + Istim) - (G)2 * INaK) + ICaK_i) * (G)k::c_myo + JdiffK * (G)(k::vss / k::vmyo);
  const G dkss = -ICaK_ss * (G)k::c_ss - JdiffK;
  const G dnai = -(INa + INaL + (G)3 * INaCa_i + ICaNa_i + (G)3 * INaK + INab) * (G)k::c_myo + JdiffNa * (G)(k::vss / k::vmyo);
  const G dnass = -(ICaNa_ss + (G)3 * INaCa_ss) * (G)k::c_ss - JdiffNa;
  const G dcass = Bcass * ((-(ICaL_ss - (G)2 * INaCa_ss) * (G)(0.5 * k::c_ss) + Jrel * (G)(k::vjsr / k::vss)) - Jdiff);
  const G dcai = Bcai * ((-((ICaL_i + IpCa + ICab) - (G)2 * INaCa_i) * (G)(0.5 * k::c_myo) - Jup * (G)(k::vnsr / k::vmyo)) +
                         Jdiff * (G)(k::vss / k::vmyo));
  const G dcansr = Jup - Jtr * (G)(k::vjsr / k::vnsr);
  const G dcajsr = Bcajsr * (Jtr - Jrel);
  const G dCaMKt = (G)k::aCaMK * CaMKb * (CaMKb + (G)y.CaMKt) - (G)k::bCaMK * (G)y.CaMKt;
  const G C1_ = (G)y.C1, C2_ = (G)y.C2, C3_ = (G)y.C3, I_ = (G)y.I, O_ = (G)y.O;
  const G dC3 = beta * C2_ - alpha * C3_;
  const G dC2 = (alpha * C3_ + (G)k::beta_1 * C1_) - (beta + (G)k::alpha_1) * C2_;
  const G dO = (alpha_2 * C1_ + beta_i * I_) - (beta_2 + alpha_i) * O_;
  const G dC1 = ((G)k::alpha_1 * C2_ + beta_2 * O_ + beta_ItoC2 * I_) - ((G)k::beta_1 + alpha_2 + alpha_C2ToI) * C1_;
  const G dI = (alpha_C2ToI * C1_ + alpha_i * O_) - (beta_ItoC2 + beta_i) * I_;
  // Rush-Larsen gates
  y.hL = rush_larsen<P, true>(y.hL, hLss, (G)k::thL, dt);
  y.hLp = rush_larsen<P, true>(y.hLp, hLssp, (G)k::thLp, dt);
  y.jca = rush_larsen<P, true>(y.jca, jcass, (G)k::tjca, dt);
  // Mixed: the Taylor form of 1 - e^{-a} for every gate whose dt/tau stays
  // small (tau >= ~0.17 ms: a <= 0.03 at dt = 0.005 ms, series error below
  // 1e-9), as the ORd family does; 1 - e^{-a} from the FP32 exponential
  // keeps only a few bits for slow gates (a ~ 5e-6). m, mL (tau down to
  // ~0.01 ms) and Jrel (tau down to 0.001 ms) keep the exponential.
  y.m = rush_larsen<P>(y.m, mss, tm, dt);
  y.mL = rush_larsen<P>(y.mL, mLss, tm, dt);
  y.a = rush_larsen<P, true>(y.a, ass, ta, dt);
  y.d = rush_larsen<P, true>(y.d, dss, td, dt);
  y.ff = rush_larsen<P, true>(y.ff, fss, tff, dt);
  y.fs = rush_larsen<P, true>(y.fs, fss, tfs, dt);
  y.xs1 = rush_larsen<P, true>(y.xs1, xs1ss, txs1, dt);
  y.ap = rush_larsen<P, true>(y.ap, assp, ta, dt);
  y.fcaf = rush_larsen<P, true>(y.fcaf, fss, tfcaf, dt);
  y.fcas = rush_larsen<P, true>(y.fcas, fss, tfcas, dt);
  y.ffp = rush_larsen<P, true>(y.ffp, fss, (G)2.5 * tff, dt);
  y.xs2 = rush_larsen<P, true>(y.xs2, xs1ss, txs2, dt);
  y.h = rush_larsen<P, true>(y.h, hss, th, dt);
  y.fcafp = rush_larsen<P, true>(y.fcafp, fss, (G)2.5 * tfcaf, dt);
  y.j = rush_larsen<P, true>(y.j, hss, tj, dt);
  y.hp = rush_larsen<P, true>(y.hp, hssp, th, dt);
  y.iF = rush_larsen<P, true>(y.iF, iss, tiF, dt);
  y.jp = rush_larsen<P, true>(y.jp, hss, (G)1.46 * tj, dt);
  y.iS = rush_larsen<P, true>(y.iS, iss, tiS, dt);
  y.iFp = rush_larsen<P, true>(y.iFp, iss, tiFp, dt);
  y.iSp = rush_larsen<P, true>(y.iSp, iss, tiSp, dt);
  y.Jrel_np = rush_larsen<P>(y.Jrel_np, Jrel_inf, tau_rel, dt);
  y.Jrel_p = rush_larsen<P>(y.Jrel_p, Jrel_infp, tau_relp, dt);
  y.nca_ss = rush_larsen<P, true>(y.nca_ss, P::dv(anca_ss * (G)k::k2n, km2n), P::rc(km2n), dt);
  y.nca_i = rush_larsen<P, true>(y.nca_i, P::dv(anca_i * (G)k::k2n, km2n), P::rc(km2n), dt);
  // forward Euler
  fe<P>(y.V, (double)dV, dt);
  fe<P>(y.CaMKt, (double)dCaMKt, dt);
  fe<P>(y.cass, (double)dcass, dt);
  fe<P>(y.nai, (double)dnai, dt);
  fe<P>(y.nass, (double)dnass, dt);
  fe<P>(y.ki, (double)dki, dt);
  fe<P>(y.kss, (double)dkss, dt);
  fe<P>(y.cansr, (double)dcansr, dt);
  fe<P>(y.cajsr, (double)dcajsr, dt);
  fe<P>(y.cai, (double)dcai, dt);
  fe<P>(y.C1, (double)dC1, dt);
  fe<P>(y.C2, (double)dC2, dt);
  fe<P>(y.C3, (double)dC3, dt);
  fe<P>(y.I, (double)dI, dt);
  fe<P>(y.O, (double)dO, dt);
}

__device__ __forceinline__ double hill_factor(double conc, double ic50, double h) {
  return (ic50 > 10E-14 && h > 10E-14) ? 1. / (1. + ::pow(conc / ic50, h)) : 1.;
}

// ___initEndo / Epi / Mid (:506-1134) and the Hill hook (:1149-1168).
__device__ __forceinline__ void init_instance(double *__restrict__ par, double *__restrict__ s_, int64_t ld,
                                              int64_t i, double ct, double conc, const double *__restrict__ hill,
                                              bool quirks) {
  const int c = ct == 1.0 ? 1 : ct == 2.0 ? 2 : 0;
  double GNa = 11.7802, GNaL = c == 1 ? 0.0279 * 0.6 : 0.0279;
  double Gto = c == 0 ? 0.16 : 0.16 * 2.0;
  double PCa = c == 1 ? 8.3757e-05 * 1.2 : c == 2 ? 8.3757e-05 * 2.0 : 8.3757e-05;
  double GKr = c == 1 ? 0.0321 * 1.3 : c == 2 ? 0.0321 * 0.8 : 0.0321;
  double GKs = c == 1 ? 0.0011 * 1.4 : 0.0011;
  double GK1 = c == 1 ? 0.6992 * 1.2 : c == 2 ? 0.6992 * 1.3 : 0.6992;
  const double GKb = c == 1 ? 0.0189 * 0.6 : 0.0189;
  const double Gncx = c == 1 ? 0.0034 * 1.1 : c == 2 ? 0.0034 * 1.4 : 0.0034;
  const double Pnak = c == 1 ? 15.4509 * 0.9 : c == 2 ? 15.4509 * 0.7 : 15.4509;
  double PCap = 1.1 * PCa, PCaNa = 0.00125 * PCa, PCaK = 0.0003574 * PCa;
  double PCaNap = 0.00125 * PCap, PCaKp = 0.0003574 * PCap;
  if (hill) {
    PCa *= hill_factor(conc, hill[0], hill[1]);
    GK1 *= hill_factor(conc, hill[2], hill[3]);
    GKs *= hill_factor(conc, hill[4], hill[5]);
    GNa *= hill_factor(conc, hill[6], hill[7]);
    GNaL *= hill_factor(conc, hill[8], hill[9]);
    Gto *= hill_factor(conc, hill[10], hill[11]);
    GKr *= hill_factor(conc, hill[12], hill[13]);
    if (!quirks) {  // the reference derives these before the block
      PCap = 1.1 * PCa; PCaNa = 0.00125 * PCa; PCaK = 0.0003574 * PCa;
      PCaNap = 0.00125 * PCap; PCaKp = 0.0003574 * PCap;
    }
  }
  const double constA = 1.82e6 * ::pow(k::dielConstant * k::T, -1.5);
  const double sIo = ::sqrt(k::Io);
  const double dh = sIo / (1.0 + sIo) - 0.3 * k::Io;
  double *p = par + i;
  p[P_GNa * ld] = GNa; p[P_GNaL * ld] = GNaL; p[P_Gto * ld] = Gto; p[P_PCa * ld] = PCa; p[P_PCap * ld] = PCap;
  p[P_PCaNa * ld] = PCaNa; p[P_PCaK * ld] = PCaK; p[P_PCaNap * ld] = PCaNap; p[P_PCaKp * ld] = PCaKp;
  p[P_GKr * ld] = GKr; p[P_GKs * ld] = GKs; p[P_GK1 * ld] = GK1; p[P_GKb * ld] = GKb; p[P_Gncx * ld] = Gncx;
  p[P_Pnak * ld] = Pnak; p[P_cmdnmax * ld] = c == 1 ? 0.05 * 1.3 : 0.05; p[P_upScale * ld] = c == 1 ? 1.3 : 1.0;
  p[P_epi * ld] = c == 1 ? 1.0 : 0.0; p[P_jrel_scale * ld] = c == 2 ? 1.7 : 1.0;
  p[P_gamma_cao * ld] = ::exp(-constA * 4.0 * dh);
  p[P_gamma_nao * ld] = ::exp(-constA * 1.0 * dh);
  p[P_gamma_ko * ld] = ::exp(-constA * 1.0 * dh);
  p[P_ECl * ld] = ((k::R * k::T) / (-1.0 * k::F)) * ::log(k::clo / k::cli);
  p[P_constA * ld] = constA;
  p[P_amp * ld] = -53; p[P_BCL * ld] = 1000; p[P_stim_start * ld] = 10; p[P_duration * ld] = 1.0;
  const double endo[kNumStates] = {
      -88.7638, 0.0111, 7.0305e-5, 12.1025, 12.1029, 142.3002, 142.3002, 1.5211, 1.5214, 8.1583e-05, 8.0572e-4,
      0.8286, 0.8284, 0.6707, 0.8281, 1.629e-4, 0.5255, 0.2872, 9.5098e-4, 0.9996, 0.5936, 4.8454e-4, 0.9996,
      0.6538, 8.1084e-9, 1.0, 0.939, 1.0, 0.9999, 1.0, 1.0, 1.0, 6.6462e-4, 0.0012, 7.0344e-4, 8.5109e-4,
      0.9981, 1.3289e-5, 3.7585e-4, 0.248, 1.7707e-4, 1.6129e-22, 1.2475e-20};
  const double epi[kNumStates] = {
      -89.1400, 0.0129, 5.7672e-05, 12.8363, 12.8366, 142.6951, 142.6951, 1.8119, 1.8102, 6.6309e-05,
      0.00074303, 0.8360, 0.8359, 0.6828, 0.8357, 0.00015166, 0.5401, 0.3034, 0.00092716, 0.9996, 0.9996,
      0.0004724, 0.9996, 0.9996, 0, 1.0, 0.9485, 1.0, 0.9999, 1.0, 1.0, 1.0, 0.00030853, 0.00053006,
      0.00067941, 0.00082869, 0.9982, 9.5416e-06, 0.00027561, 0.2309, 0.00016975, 2.8189e-24, 0};
  const double mid[kNumStates] = {
      -89.1704, 0.0192, 6.5781e-05, 15.0038, 15.0043, 143.0403, 143.0402, 1.9557, 1.9593, 8.166e-05,
      0.00073818, 0.8365, 0.8363, 0.6838, 0.8358, 0.00015079, 0.5327, 0.2834, 0.00092527, 0.9996, 0.5671,
      0.00047143, 0.9996, 0.6261, 0, 1.0, 0.92, 1.0, 0.9998, 1.0, 1.0, 1.0, 0.00051399, 0.0012, 0.00069560,
      0.00082672, 0.9979, 1.8784e-05, 0.00054206, 0.2653, 0.00016921, 0, 0};
  const double *y0 = c == 1 ? epi : c == 2 ? mid : endo;
#pragma unroll 1
  for (int k2 = 0; k2 < kNumStates; ++k2) s_[k2 * ld + i] = y0[k2];
}

}  // namespace tomek
}  // namespace cep
