// ten Tusscher 2006 epicardial model (IK1 Ko-dependent variant), one cell
// per thread, templated on the precision policy (cep_device.cuh).
//
// Equations and update scheme: CEPCell_NEO/cellmodels/
// ten_tusscher_model_2006_IK1Ko_epi_units.cpp computeRates (:274-380) and
// solveAnalytical (:382-407): Rush-Larsen for the 12 gates, forward Euler
// for V, the ions and R'. The stimulus is the reference's periodic
// single-cell form (:335-337) or the tissue flag isS1 (:338-345). The drug
// hook (absent from the reference model) follows the reference's TT2004 one
// (tentusscher_noble_noble_panfilov_2004_b.cpp:361-377).
#pragma once
#include "cep_device.cuh"

namespace cep {
namespace tt06 {

constexpr int kNumStates = 19;
enum : int { V = 0, K_i, Na_i, Ca_i, Xr1, Xr2, Xs, m, h, j, Ca_ss, d, f, f2, fCass, s, r, Ca_SR, R_prime };
enum : int {
  P_gCaL = 0, P_gK1, P_gKs, P_gNa, P_gto, P_gKr, P_amp, P_BCL, P_stim_start, P_duration,
  P_gbna, P_gbca, P_gpCa, P_gpK,  // background and pump conductances (scalable per instance)
  kNumParams
};

namespace k {
constexpr double R = 8314.472, T = 310, F = 96485.3415, Cm = 0.185, V_c = 0.016404, P_kna = 0.03, K_o = 5.4;
constexpr double Na_o = 140, Ca_o = 2, g_bna = 0.00029, g_bca = 0.000592, P_NaK = 2.724, K_mk = 1, K_mNa = 40;
constexpr double K_NaCa = 1000, K_sat = 0.1, alpha = 2.5, gmma = 0.35, Km_Ca = 1.38, Km_Nai = 87.5;
constexpr double g_pCa = 0.1238, K_pCa = 0.0005, g_pK = 0.0146, k1_prime = 0.15, k2_prime = 0.045, k3 = 0.06;
constexpr double k4 = 0.005, EC = 1.5, max_sr = 2.5, min_sr = 1, V_rel = 0.102, V_xfer = 0.0038, K_up = 0.00025;
constexpr double V_leak = 0.00036, Vmax_up = 0.006375, Buf_c = 0.2, K_buf_c = 0.001, Buf_sr = 10, K_buf_sr = 0.3;
constexpr double Buf_ss = 0.4, K_buf_ss = 0.00025, V_sr = 0.001094, V_ss = 0.00005468;
constexpr double RTF = (R * T) / F, FRT = F / (R * T);
constexpr double nak_c = (P_NaK * K_o) / (K_o + K_mk);
constexpr double naca_den = (Km_Nai * Km_Nai * Km_Nai + Na_o * Na_o * Na_o) * (Km_Ca + Ca_o);
constexpr double Na_o3 = Na_o * Na_o * Na_o;
constexpr double c_vcf = Cm / (V_c * F);  // current -> concentration rate
}  // namespace k

template <class G>
struct Y {
  double V, K_i, Na_i, Ca_i, Xr1, Xr2, Xs, m, h, j, Ca_ss, d, f, f2, fCass, s, r, Ca_SR, R_prime;
};
template <class G>
struct Par {
  G gCaL, gK1, gKs, gNa, gto, gKr;
  double amp, BCL, stim_start, duration;
  G gbna, gbca, gpCa, gpK;
};
template <class G>
struct Cur {
  G INa, INaL, Ito, ICaL, IKr, IKs, IK1, dVdt;
};

#define CEP_TT_FIELDS(X) X(V) X(K_i) X(Na_i) X(Ca_i) X(Xr1) X(Xr2) X(Xs) X(m) X(h) X(j) X(Ca_ss) X(d) X(f) \
  X(f2) X(fCass) X(s) X(r) X(Ca_SR) X(R_prime)

template <class G>
__device__ __forceinline__ void load(Y<G> &y, const double *__restrict__ s_, int64_t ld, int64_t i) {
#define CEP_LD(n) y.n = s_[n * ld + i];
  CEP_TT_FIELDS(CEP_LD)
#undef CEP_LD
}
template <class G>
__device__ __forceinline__ void store(const Y<G> &y, double *__restrict__ s_, int64_t ld, int64_t i) {
#define CEP_ST(n) s_[n * ld + i] = y.n;
  CEP_TT_FIELDS(CEP_ST)
#undef CEP_ST
}
template <class G>
__device__ __forceinline__ void load_par(Par<G> &q, const double *__restrict__ p, int64_t ld, int64_t i) {
  q.gCaL = (G)p[P_gCaL * ld + i]; q.gK1 = (G)p[P_gK1 * ld + i]; q.gKs = (G)p[P_gKs * ld + i];
  q.gNa = (G)p[P_gNa * ld + i]; q.gto = (G)p[P_gto * ld + i]; q.gKr = (G)p[P_gKr * ld + i];
  q.amp = p[P_amp * ld + i]; q.BCL = p[P_BCL * ld + i]; q.stim_start = p[P_stim_start * ld + i];
  q.duration = p[P_duration * ld + i];
  q.gbna = (G)p[P_gbna * ld + i]; q.gbca = (G)p[P_gbca * ld + i]; q.gpCa = (G)p[P_gpCa * ld + i];
  q.gpK = (G)p[P_gpK * ld + i];
}

// One cell step: rates at (t, y); if `update`, the reference's Rush-Larsen /
// forward-Euler update by dt. stim_mode < 0: periodic single-cell stimulus;
// 0/1: the tissue flag.
template <class P>
__device__ __forceinline__ void step(Y<typename P::G> &y, const Par<typename P::G> &q, double t, double dt,
                                     int stim_mode, bool update, Cur<typename P::G> &cur) {
  using G = typename P::G;
  const G v = (G)y.V, one = (G)1;
  bool on;
  if (stim_mode < 0) {
    const double ph = t - floor(t / q.BCL) * q.BCL;
    on = ph >= q.stim_start && ph <= q.stim_start + q.duration;
  } else {
    on = stim_mode != 0;
  }
  const G i_Stim = on ? -(G)q.amp : (G)0;
  const G f_inf = P::rc(one + P::ex((v + (G)20.0) * (G)(1.0 / 7.0)));
  const G tau_f = (G)1102.5 * P::ex(-p2(v + (G)27.0) * (G)(1.0 / 225.0)) + P::dv((G)200.0, one + P::ex(((G)13.0 - v) * (G)0.1)) +
                  P::dv((G)180.0, one + P::ex((v + (G)30.0) * (G)0.1)) + (G)20.0;
  const G f2_inf = P::dv((G)0.67, one + P::ex((v + (G)35.0) * (G)(1.0 / 7.0))) + (G)0.33;
  const G tau_f2 = (G)562.0 * P::ex(-p2(v + (G)27.0) * (G)(1.0 / 240.0)) + P::dv((G)31.0, one + P::ex(((G)25.0 - v) * (G)0.1)) +
                   P::dv((G)80.0, one + P::ex((v + (G)30.0) * (G)0.1));
  const G cass_g = (G)y.Ca_ss, cai_g = (G)y.Ca_i, casr_g = (G)y.Ca_SR;
  const G cass2 = p2(cass_g * (G)20.0);  // (Ca_ss / 0.05)^2
  const G fCass_inf = P::dv((G)0.6, one + cass2) + (G)0.4;
  const G tau_fCass = P::dv((G)80.0, one + cass2) + (G)2.0;
  const G s_inf = P::rc(one + P::ex((v + (G)20.0) * (G)0.2));
  const G tau_s = (G)85.0 * P::ex(-p2(v + (G)45.0) * (G)(1.0 / 320.0)) + P::dv((G)5.0, one + P::ex((v - (G)20.0) * (G)0.2)) + (G)3.0;
  const G r_inf = P::rc(one + P::ex(((G)20.0 - v) * (G)(1.0 / 6.0)));
  const G tau_r = (G)9.5 * P::ex(-p2(v + (G)40.0) * (G)(1.0 / 1800.0)) + (G)0.8;
  const G xr1_inf = P::rc(one + P::ex(((G)-26.0 - v) * (G)(1.0 / 7.0)));
  const G tau_xr1 = P::dv((G)450.0, one + P::ex(((G)-45.0 - v) * (G)0.1)) * P::dv((G)6.0, one + P::ex((v + (G)30.0) * (G)(1.0 / 11.5)));
  const G xr2_inf = P::rc(one + P::ex((v + (G)88.0) * (G)(1.0 / 24.0)));
  const G tau_xr2 = P::dv((G)3.0, one + P::ex(((G)-60.0 - v) * (G)0.05)) * P::dv((G)1.12, one + P::ex((v - (G)60.0) * (G)0.05));
  const G xs_inf = P::rc(one + P::ex(((G)-5.0 - v) * (G)(1.0 / 14.0)));
  const G tau_xs = P::dv((G)1400.0, P::sq(one + P::ex(((G)5.0 - v) * (G)(1.0 / 6.0)))) * P::rc(one + P::ex((v - (G)35.0) * (G)(1.0 / 15.0))) + (G)80.0;
  const G m_inf = P::rc(p2(one + P::ex(((G)-56.86 - v) * (G)(1.0 / 9.03))));
  const G tau_m = P::rc(one + P::ex(((G)-60.0 - v) * (G)0.2)) *
                  (P::dv((G)0.1, one + P::ex((v + (G)35.0) * (G)0.2)) + P::dv((G)0.1, one + P::ex((v - (G)50.0) * (G)0.005)));
  const G h_inf = P::rc(p2(one + P::ex((v + (G)71.55) * (G)(1.0 / 7.43))));
  const bool lo = v < (G)-40.0;
  const G alpha_h = lo ? (G)0.057 * P::ex(-(v + (G)80.0) * (G)(1.0 / 6.8)) : (G)0;
  const G beta_h = lo ? (G)2.7 * P::ex((G)0.079 * v) + (G)310000.0 * P::ex((G)0.3485 * v)
                      : P::dv((G)0.77, (G)0.13 * (one + P::ex((v + (G)10.66) * (G)(1.0 / -11.1))));
  const G tau_h = P::rc(alpha_h + beta_h);
  const G j_inf = h_inf;
  const G alpha_j = lo ? P::dv(((G)-25428.0 * P::ex((G)0.2444 * v) - (G)6.948e-06 * P::ex((G)-0.04391 * v)) * (v + (G)37.78),
                               one + P::ex((G)0.311 * (v + (G)79.23)))
                       : (G)0;
  const G beta_j = lo ? P::dv((G)0.02424 * P::ex((G)-0.01052 * v), one + P::ex((G)-0.1378 * (v + (G)40.14)))
                      : P::dv((G)0.6 * P::ex((G)0.057 * v), one + P::ex((G)-0.1 * (v + (G)32.0)));
  const G tau_j = P::rc(alpha_j + beta_j);
  const G d_inf = P::rc(one + P::ex(((G)-8.0 - v) * (G)(1.0 / 7.5)));
  const G tau_d = (P::dv((G)1.4, one + P::ex(((G)-35.0 - v) * (G)(1.0 / 13.0))) + (G)0.25) *
                      P::dv((G)1.4, one + P::ex((v + (G)5.0) * (G)0.2)) +
                  P::rc(one + P::ex(((G)50.0 - v) * (G)0.05));
  const G nai_g = (G)y.Na_i, ki_g = (G)y.K_i;
  const G i_NaK = P::dv((G)k::nak_c * nai_g, nai_g + (G)k::K_mNa) *
                  P::rc(one + (G)0.1245 * P::ex((G)-0.1 * v * (G)k::FRT) + (G)0.0353 * P::ex(-v * (G)k::FRT));
  const G E_Na = (G)k::RTF * P::lg(P::dv((G)k::Na_o, nai_g));
  const G i_Na = q.gNa * p3((G)y.m) * (G)y.h * (G)y.j * (v - E_Na);
  const G i_b_Na = q.gbna * (v - E_Na);
  const G eg = P::ex((G)k::gmma * v * (G)k::FRT), eg1 = P::ex(((G)k::gmma - one) * v * (G)k::FRT);
  const G i_NaCa = P::dv((G)k::K_NaCa * (eg * p3(nai_g) * (G)k::Ca_o - eg1 * (G)k::Na_o3 * cai_g * (G)k::alpha),
                         (G)k::naca_den * (one + (G)k::K_sat * eg1));
  const G E_K = (G)k::RTF * P::lg(P::dv((G)k::K_o, ki_g));
  const G vek = v - E_K;
  const G alpha_K1 = P::dv((G)0.1, one + P::ex((G)0.06 * (vek - (G)200.0)));
  const G beta_K1 = P::dv((G)3.0 * P::ex((G)0.0002 * (vek + (G)100.0)) + P::ex((G)0.1 * (vek - (G)10.0)),
                          one + P::ex((G)-0.5 * vek));
  const G i_K1 = q.gK1 * P::dv(alpha_K1, alpha_K1 + beta_K1) * vek;  // sqrt(K_o/5.4) = 1
  const G i_to = q.gto * (G)y.r * (G)y.s * vek;
  const G i_Kr = q.gKr * (G)y.Xr1 * (G)y.Xr2 * vek;
  const G E_Ks = (G)k::RTF * P::lg(P::dv((G)(k::K_o + k::P_kna * k::Na_o), ki_g + (G)k::P_kna * nai_g));
  const G i_Ks = q.gKs * p2((G)y.Xs) * (v - E_Ks);
  G i_CaL;
  if constexpr (P::kMixed) {
    const G x = (G)2.0 * (v - (G)15.0) * (G)k::FRT;
    const G e = P::ex(x);
    // g d f f2 fCass 4 (V-15) F^2/(RT) (0.25 Ca_ss e - Ca_o)/(e - 1) with the
    // x/(e^x - 1) factor evaluated stably
    i_CaL = q.gCaL * (G)y.d * (G)y.f * (G)y.f2 * (G)y.fCass * (G)(2.0 * k::F) * ghk_factor(x) *
            ((G)0.25 * cass_g * e - (G)k::Ca_o);
  } else {
    const double vv = y.V;
    const double e = exp_f64((2.0 * (vv - 15.0) * k::F) / (k::R * k::T));
    i_CaL = div64(((q.gCaL * y.d * y.f * y.f2 * y.fCass * 4.0 * (vv - 15.0) * (k::F * k::F)) / (k::R * k::T)) *
                      (0.25 * y.Ca_ss * e - k::Ca_o),
                  e - 1.0);
  }
  const G E_Ca = (G)(0.5 * k::RTF) * P::lg(P::dv((G)k::Ca_o, cai_g));
  const G i_b_Ca = q.gbca * (v - E_Ca);
  const G i_p_K = P::dv(q.gpK * vek, one + P::ex(((G)25.0 - v) * (G)(1.0 / 5.98)));
  const G i_p_Ca = P::dv(q.gpCa * cai_g, cai_g + (G)k::K_pCa);
  const G dV = -(i_K1 + i_to + i_Kr + i_Ks + i_CaL + i_NaK + i_Na + i_b_Na + i_NaCa + i_b_Ca + i_p_K + i_p_Ca + i_Stim);
  cur.INa = i_Na; cur.INaL = (G)0; cur.Ito = i_to; cur.ICaL = i_CaL; cur.IKr = i_Kr; cur.IKs = i_Ks;
  cur.IK1 = i_K1; cur.dVdt = dV;
  if (!update) return;
  const G i_up = P::dv((G)k::Vmax_up, one + P::dv((G)(k::K_up * k::K_up), p2(cai_g)));
  const G i_leak = (G)((y.Ca_SR - y.Ca_i) * k::V_leak);
  const G i_xfer = (G)((y.Ca_ss - y.Ca_i) * k::V_xfer);
  const G Ca_i_bufc = P::rc(one + P::dv((G)(k::Buf_c * k::K_buf_c), p2(cai_g + (G)k::K_buf_c)));
  const G kcasr = (G)k::max_sr - P::dv((G)(k::max_sr - k::min_sr), one + p2(P::dv((G)k::EC, casr_g)));
  const G k2 = (G)k::k2_prime * kcasr;
  const G k1 = P::dv((G)k::k1_prime, kcasr);
  const G O = P::dv(k1 * p2(cass_g) * (G)y.R_prime, (G)k::k3 + k1 * p2(cass_g));
  const G i_rel = (G)k::V_rel * O * (G)(y.Ca_SR - y.Ca_ss);
  const G Ca_sr_bufsr = P::rc(one + P::dv((G)(k::Buf_sr * k::K_buf_sr), p2(casr_g + (G)k::K_buf_sr)));
  const G Ca_ss_bufss = P::rc(one + P::dv((G)(k::Buf_ss * k::K_buf_ss), p2(cass_g + (G)k::K_buf_ss)));
  const G dNa_i = -(i_Na + i_b_Na + (G)3.0 * i_NaK + (G)3.0 * i_NaCa) * (G)k::c_vcf;
  const G dK_i = -((i_K1 + i_to + i_Kr + i_Ks + i_p_K + i_Stim) - (G)2.0 * i_NaK) * (G)k::c_vcf;
  const G dCa_i = Ca_i_bufc * ((((i_leak - i_up) * (G)(k::V_sr / k::V_c)) + i_xfer) -
                               ((i_b_Ca + i_p_Ca) - (G)2.0 * i_NaCa) * (G)(0.5 * k::c_vcf));
  const G dR = -k2 * cass_g * (G)y.R_prime + (G)k::k4 * (one - (G)y.R_prime);
  const G dCa_SR = Ca_sr_bufsr * (i_up - (i_rel + i_leak));
  const G dCa_ss = Ca_ss_bufss * ((-i_CaL * (G)(k::Cm / (2.0 * k::V_ss * k::F)) + i_rel * (G)(k::V_sr / k::V_ss)) -
                                  i_xfer * (G)(k::V_c / k::V_ss));
  // Rush-Larsen gates (the reference's ((y - inf) e^{-dt/tau}) + inf)
  if constexpr (P::kMixed) {
    y.f = rush_larsen<P, true>(y.f, f_inf, tau_f, dt);
    y.f2 = rush_larsen<P, true>(y.f2, f2_inf, tau_f2, dt);
    y.fCass = rush_larsen<P, true>(y.fCass, fCass_inf, tau_fCass, dt);
    y.s = rush_larsen<P, true>(y.s, s_inf, tau_s, dt);
    y.r = rush_larsen<P>(y.r, r_inf, tau_r, dt);
    y.Xr1 = rush_larsen<P>(y.Xr1, xr1_inf, tau_xr1, dt);
    y.Xr2 = rush_larsen<P>(y.Xr2, xr2_inf, tau_xr2, dt);
    y.Xs = rush_larsen<P, true>(y.Xs, xs_inf, tau_xs, dt);
    y.m = rush_larsen<P>(y.m, m_inf, tau_m, dt);
    y.h = rush_larsen<P>(y.h, h_inf, tau_h, dt);
    y.j = rush_larsen<P>(y.j, j_inf, tau_j, dt);
    y.d = rush_larsen<P>(y.d, d_inf, tau_d, dt);
  } else {
#define CEP_RL(n, inf, tau) y.n = ((y.n - (inf)) * exp_f64(div64(-dt, (tau)))) + (inf);
    CEP_RL(f, f_inf, tau_f) CEP_RL(f2, f2_inf, tau_f2) CEP_RL(fCass, fCass_inf, tau_fCass) CEP_RL(s, s_inf, tau_s)
    CEP_RL(r, r_inf, tau_r) CEP_RL(Xr1, xr1_inf, tau_xr1) CEP_RL(Xr2, xr2_inf, tau_xr2) CEP_RL(Xs, xs_inf, tau_xs)
    CEP_RL(m, m_inf, tau_m) CEP_RL(h, h_inf, tau_h) CEP_RL(j, j_inf, tau_j) CEP_RL(d, d_inf, tau_d)
#undef CEP_RL
  }
  y.V = y.V + (double)dV * dt;
  y.R_prime = y.R_prime + (double)dR * dt;
  y.Na_i = y.Na_i + (double)dNa_i * dt;
  y.K_i = y.K_i + (double)dK_i * dt;
  y.Ca_SR = y.Ca_SR + (double)dCa_SR * dt;
  y.Ca_ss = y.Ca_ss + (double)dCa_ss * dt;
  y.Ca_i = y.Ca_i + (double)dCa_i * dt;
}

__device__ __forceinline__ double hill_factor(double conc, double ic50, double h) {
  return (ic50 > 10E-14 && h > 10E-14) ? 1. / (1. + ::pow(conc / ic50, h)) : 1.;
}

// initConsts (:196-272) plus the Hill block of g_CaL, g_K1, g_Ks, g_Na, g_to,
// g_Kr (reference CSV columns 0-7, 10-13).
__device__ __forceinline__ void init_instance(double *__restrict__ par, double *__restrict__ s_, int64_t ld,
                                              int64_t i, double conc, const double *__restrict__ hill) {
  double gCaL = 0.0000398, gK1 = 5.405, gKs = 0.392, gNa = 14.838, gto = 0.294, gKr = 0.153;
  if (hill) {
    gCaL *= hill_factor(conc, hill[0], hill[1]);
    gK1 *= hill_factor(conc, hill[2], hill[3]);
    gKs *= hill_factor(conc, hill[4], hill[5]);
    gNa *= hill_factor(conc, hill[6], hill[7]);
    gto *= hill_factor(conc, hill[10], hill[11]);
    gKr *= hill_factor(conc, hill[12], hill[13]);
  }
  double *p = par + i;
  p[P_gCaL * ld] = gCaL; p[P_gK1 * ld] = gK1; p[P_gKs * ld] = gKs; p[P_gNa * ld] = gNa; p[P_gto * ld] = gto;
  p[P_gKr * ld] = gKr; p[P_amp * ld] = 52; p[P_BCL * ld] = 1000; p[P_stim_start * ld] = 10; p[P_duration * ld] = 1;
  p[P_gbna * ld] = k::g_bna; p[P_gbca * ld] = k::g_bca; p[P_gpCa * ld] = k::g_pCa; p[P_gpK * ld] = k::g_pK;
  const double y0[kNumStates] = {-85.23, 136.89, 8.604, 0.000126, 0.00621, 0.4712, 0.0095, 0.00172, 0.7444, 0.7045,
                                 0.00036, 3.373e-5, 0.7888, 0.9755, 0.9953, 0.999998, 2.42e-8, 3.64, 0.9073};
#pragma unroll
  for (int k2 = 0; k2 < kNumStates; ++k2) s_[k2 * ld + i] = y0[k2];
}

}  // namespace tt06
}  // namespace cep
