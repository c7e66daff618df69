// Shared device-side definitions for the ionic-model kernels.
//
// Two precision policies drive every model template:
//   F64   - plain FP64 path: every quantity in double, CUDA's double exp/log
//           (<= 1 ulp); the ORd family takes the algebraic rewrites below
//           (CEP_F64_REWRITES), the other models the reference's forms.
//   Mixed - gates, rate constants and channel currents in FP32 with SFU
//           exp/log (ex2.approx / lg2.approx) and approximate division; the
//           membrane voltage, the ionic concentrations, CaMKII and every
//           accumulation stay FP64.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace cep {

// Reciprocal in FP64 by Newton-Raphson refinement of the hardware's 20-bit
// reciprocal seed (rcp.approx.ftz.f64): two steps r <- r + r(1 - x r) give
// a result within about an ulp for 2^-1021 <= |x| <= 2^1021. Outside that
// range the seed is flushed or infinite and the steps end in NaN (zero,
// subnormal, infinite or NaN x), which the callers below send to an exact
// special-case path.
__device__ __forceinline__ double rcp64_nr(double x) {
  double r;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
  double e = fma(-x, r, 1.0);
  r = fma(r, e, r);
  e = fma(-x, r, 1.0);
  return fma(r, e, r);
}
// 1/x for x = +-0 (+-inf), +-inf (+-0), NaN, and subnormal x, scaled by
// 2^64 into the normal range (the result overflows to inf as IEEE's does
// when |x| < 2^-1024).
__device__ __noinline__ double rcp64_special(double x) {
  if (isnan(x)) return x;
  if (x == 0.0) return copysign(INFINITY, x);
  if (isinf(x)) return copysign(0.0, x);
  return rcp64_nr(x * 0x1p64) * 0x1p64;
}
__device__ __forceinline__ double rcp64(double x) {
  const double r = rcp64_nr(x);
  return isnan(r) ? rcp64_special(x) : r;
}
// a / b for the operands the fast path turns into NaN: NaN operands, zero,
// subnormal or infinite divisors, infinite dividends and quotients that
// overflow. Finite cases divide the frexp mantissas and scale the result
// back with ldexp (one extra rounding for subnormal quotients).
__device__ __noinline__ double div64_special(double a, double b) {
  if (isnan(a) || isnan(b)) return a + b;
  const bool neg = signbit(a) != signbit(b);
  if (isinf(b)) return isinf(a) ? NAN : (neg ? -0.0 : 0.0);
  if (b == 0.0) return a == 0.0 ? NAN : (neg ? -INFINITY : INFINITY);
  if (isinf(a)) return neg ? -INFINITY : INFINITY;
  if (a == 0.0) return neg ? -0.0 : 0.0;
  int ea, eb;
  const double ma = frexp(a, &ea), mb = frexp(b, &eb);
  const double r = rcp64_nr(mb);
  const double q = ma * r;
  return ldexp(fma(r, fma(-mb, q, ma), q), ea - eb);
}
// a / b as a * (1/b) with one residual correction (q + r (a - b q)), within
// an ulp of the correctly rounded quotient for divisors of magnitude up to
// 2^1021 (every division of the models here); IEEE results for zero,
// subnormal, infinite and NaN operands. 1/b takes one Newton-Raphson step
// from the seed (relative error e^2 for a seed error e <= 2^-20), which the
// correction squares again: q + r (a - b q) = (a/b)(1 - e^4) up to the
// roundings of q and of the result. Zero, subnormal and infinite divisors
// end in NaN as in rcp64_nr.
__device__ __forceinline__ double div64(double a, double b) {
  double r;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(b));
  r = fma(r, fma(-b, r, 1.0), r);
  const double q = a * r;
  const double out = fma(r, fma(-b, q, a), q);
  return isnan(out) ? div64_special(a, b) : out;
}

// FP64 takes the same algebraic rewrites as the mixed policy (rate-form
// time constants, shared exponentials, log differences, shared reciprocals:
// model_ord.cuh) and the series of e^{-a} for slow gates with a < 0.1; each
// changes a result by a few ulp, far inside the FP64 path's bound against
// the reference (1e-6 mV). Building with -DCEP_F64_REWRITES=0 restores the
// reference's written forms.
#ifndef CEP_F64_REWRITES
#define CEP_F64_REWRITES 1
#endif

// CUDA's double exp and log called out of line: each inlined copy is a few
// dozen instructions, and the ORd family's FP64 step calls them ~130 times,
// which made the step's code too large for the instruction caches
// (no_instruction stalls 6 cycles per issued instruction in the 2-warp form);
// one shared copy of each keeps it resident (about 2x the FP64 throughput).
__device__ __noinline__ double exp_f64(double x) { return ::exp(x); }
__device__ __noinline__ double log_f64(double x) { return ::log(x); }

// Two exponentials of independent arguments in one out-of-line body, where
// the two instruction streams interleave: one call's latency for two
// results (the ORd family's time constants are sums of two exponentials).
__device__ __noinline__ double2 exp2_f64(double a, double b) { return make_double2(::exp(a), ::exp(b)); }

template <class G>
struct Exp2 {
  G a, b;
};
// Four exponentials of independent arguments in one out-of-line body: the
// steady states of a channel group are each a logistic of V, and one call
// overlaps their four dependency chains.
struct Dbl4 {
  double a, b, c, d;
};
__device__ __noinline__ __attribute__((const)) Dbl4 exp4_f64(double a, double b, double c, double d) {
  return Dbl4{::exp(a), ::exp(b), ::exp(c), ::exp(d)};
}
// A group of independent exponentials read through a(), b(), ...: FP64
// evaluates them together in one out-of-line call (their chains overlap);
// the mixed path evaluates each SFU exponential where it is read, so the
// grouping does not hold FP32 results in registers across the code.
struct GrpD {
  double v[4];
  __device__ __forceinline__ double a() const { return v[0]; }
  __device__ __forceinline__ double b() const { return v[1]; }
  __device__ __forceinline__ double c() const { return v[2]; }
  __device__ __forceinline__ double d() const { return v[3]; }
};
struct GrpF {
  float x[4];
  __device__ __forceinline__ float a() const { return __expf(x[0]); }
  __device__ __forceinline__ float b() const { return __expf(x[1]); }
  __device__ __forceinline__ float c() const { return __expf(x[2]); }
  __device__ __forceinline__ float d() const { return __expf(x[3]); }
};

struct F64 {
  using G = double;
  static constexpr bool kMixed = false;
  static constexpr bool kFast = CEP_F64_REWRITES != 0;
  static constexpr bool kRates = false;
  __device__ __forceinline__ static double ex(double x) { return exp_f64(x); }
  __device__ __forceinline__ static double lg(double x) { return log_f64(x); }
  __device__ __forceinline__ static Exp2<double> ex2(double a, double b) {
    const double2 r = exp2_f64(a, b);
    return {r.x, r.y};
  }
  __device__ __forceinline__ static GrpD grp4(double a, double b, double c, double d) {
    const Dbl4 r = exp4_f64(a, b, c, d);
    return GrpD{{r.a, r.b, r.c, r.d}};
  }
  __device__ __forceinline__ static GrpD grp2(double a, double b) {
    const double2 r = exp2_f64(a, b);
    return GrpD{{r.x, r.y, 0.0, 0.0}};
  }
  __device__ __forceinline__ static double dv(double a, double b) { return div64(a, b); }
  __device__ __forceinline__ static double rc(double x) { return rcp64(x); }
  // x^y for x > 0 as exp(y log x) (the exponents here are constants of
  // order 1, so the error stays at a few ulp)
  __device__ __forceinline__ static double pw(double x, double y) { return exp_f64(y * log_f64(x)); }
  __device__ __forceinline__ static double sq(double x) { return ::sqrt(x); }
};

struct Mixed {
  using G = float;
  static constexpr bool kMixed = true;
  static constexpr bool kFast = true;
  static constexpr bool kRates = false;
  __device__ __forceinline__ static float ex(float x) { return __expf(x); }
  __device__ __forceinline__ static float lg(float x) { return __logf(x); }
  __device__ __forceinline__ static Exp2<float> ex2(float a, float b) { return {__expf(a), __expf(b)}; }
  __device__ __forceinline__ static GrpF grp4(float a, float b, float c, float d) { return GrpF{{a, b, c, d}}; }
  __device__ __forceinline__ static GrpF grp2(float a, float b) { return GrpF{{a, b, 0.f, 0.f}}; }
  __device__ __forceinline__ static float dv(float a, float b) { return __fdividef(a, b); }
  __device__ __forceinline__ static float rc(float x) { return __fdividef(1.0f, x); }
  __device__ __forceinline__ static float pw(float x, float y) { return __powf(x, y); }
  __device__ __forceinline__ static float sq(float x) { return sqrtf(x); }
};

// FP64 with every update of a step replaced by the state's right-hand side:
// after one step in this policy the state array holds the model's RATES
// (a gate's (y_inf - y)/tau, the forward-Euler derivative of every other
// state), as computeRates fills them for an ODE solver (the reference
// integrates CiPA-ORd and ToR-ORd with CVODE through computeRates,
// CEPCell_NEO/modules/commons.cpp:26-35).
struct F64Rates : F64 {
  static constexpr bool kRates = true;
};

// Forward-Euler update y += d dt, or y = d (the rate) under F64Rates.
template <class P>
__device__ __forceinline__ void fe(double &y, double d, double dt) {
  if constexpr (P::kRates) y = d;
  else y = y + d * dt;
}

// c1 e^{x1} + c2 e^{x2} with both exponentials from one paired evaluation
template <class P>
__device__ __forceinline__ typename P::G esum(typename P::G c1, typename P::G x1, typename P::G c2, typename P::G x2) {
  const auto e = P::ex2(x1, x2);
  return c1 * e.a + c2 * e.b;
}

// x^2, x^3, x^4, x^8 by repeated products (the reference calls pow() with
// integral exponents; products differ from a correctly rounded pow by at
// most an ulp).
template <class T> __device__ __forceinline__ T p2(T x) { return x * x; }
template <class T> __device__ __forceinline__ T p3(T x) { return x * x * x; }
template <class T> __device__ __forceinline__ T p4(T x) { T y = x * x; return y * y; }
template <class T> __device__ __forceinline__ T p8(T x) { T y = x * x; y = y * y; return y * y; }

// x / (e^x - 1), the Goldman-Hodgkin-Katz factor, evaluated without the
// cancellation the direct form suffers for |x| -> 0 (series below 1e-3);
// ghk_factor_e takes e = e^x already at hand.
__device__ __forceinline__ float ghk_factor_e(float x, float e) {
  if (fabsf(x) < 1e-3f) return 1.0f - 0.5f * x + x * x * (1.0f / 12.0f);
  return __fdividef(x, e - 1.0f);
}
__device__ __forceinline__ float ghk_factor(float x) {
  if (fabsf(x) < 1e-3f) return 1.0f - 0.5f * x + x * x * (1.0f / 12.0f);
  return __fdividef(x, __expf(x) - 1.0f);
}

// e^{-a} for 0 <= a < 0.1 from its Taylor series to degree 10 (Horner):
// the remainder a^11/11! is below 2.6e-19, under FP64 rounding.
__device__ __forceinline__ double exp_neg_series(double a) {
  double s = 1.0 / 3628800.0;
  s = fma(s, -a, 1.0 / 362880.0);
  s = fma(s, -a, 1.0 / 40320.0);
  s = fma(s, -a, 1.0 / 5040.0);
  s = fma(s, -a, 1.0 / 720.0);
  s = fma(s, -a, 1.0 / 120.0);
  s = fma(s, -a, 1.0 / 24.0);
  s = fma(s, -a, 1.0 / 6.0);
  s = fma(s, -a, 0.5);
  s = fma(s, -a, 1.0);
  return fma(s, -a, 1.0);
}

// Rush-Larsen update of a gate whose state is kept in FP64.
//   F64  : y_inf - (y_inf - y) * exp(-dt/tau), the reference's form.
//   Mixed: y + (y_inf - y) * (1 - exp(-dt/tau)) with the increment formed in
//          FP32 and accumulated in FP64. At dt = 0.005 ms a gate with a time
//          constant of a second changes by ~1e-7 per step, below FP32
//          resolution of the state itself, so only the increment is FP32.
//          `slow` gates (tau >= 0.5 ms everywhere) take 1 - e^-a from its
//          Taylor series (a <= 0.01: relative error < 1e-10); the others
//          from the SFU exponential.
template <class P, bool slow = false>
__device__ __forceinline__ double rush_larsen(double y, typename P::G yinf, typename P::G tau, double dt) {
  using G = typename P::G;
  if constexpr (P::kMixed) {
    const G a = P::dv((G)dt, tau);
    G f;
    if constexpr (slow)
      f = a * ((G)1 - a * ((G)0.5 - a * ((G)(1.0 / 6.0) - a * (G)(1.0 / 24.0))));
    else
      f = (G)1 - P::ex(-a);
    return y + (double)((yinf - (G)y) * f);
  } else if constexpr (P::kRates) {
    return div64(yinf - y, tau);
  } else if constexpr (P::kFast && slow) {
    const double a = div64(dt, tau);
    return yinf - (yinf - y) * (a < 0.1 ? exp_neg_series(a) : exp_f64(-a));
  } else {
    return yinf - (yinf - y) * exp_f64(div64(-dt, tau));
  }
}

// A gate's time constant in the form each policy integrates with. With the
// written forms (CEP_F64_REWRITES=0) F64 keeps tau itself, computed as the
// reference writes it, for exp(-dt/tau). Otherwise both policies keep the
// rate 1/tau: where tau is a quotient num/sum of the model's rate
// terms, a = dt*sum/num needs no SFU reciprocal or division (two dependent
// MUFU ops fewer per gate).
template <class P>
struct Tau {
  typename P::G v;
};
// tau = num / sum (num a constant; 1/sum when num == 1)
template <class P>
__device__ __forceinline__ Tau<P> tau_quot(double num, typename P::G sum) {
  using G = typename P::G;
  if constexpr (P::kFast) {
    if (num == 1.0) return {sum};
    return {sum * (G)(1.0 / num)};
  } else {
    return {num == 1.0 ? P::rc(sum) : P::dv((G)num, sum)};
  }
}
// tau * s (s a constant)
template <class P>
__device__ __forceinline__ Tau<P> tau_scaled(Tau<P> t, double s) {
  using G = typename P::G;
  if constexpr (P::kFast) return {t.v * (G)(1.0 / s)};
  else return {(G)s * t.v};
}
// tau = (c + 1/sum) * s (c a constant, s = 1 unless given): F64 as written;
// Mixed 1/tau = sum / ((c sum + 1) s), one SFU division for the two the
// written form takes
template <class P>
__device__ __forceinline__ Tau<P> tau_affine(double c, typename P::G sum, typename P::G s = (typename P::G)1) {
  using G = typename P::G;
  if constexpr (P::kFast) return {P::dv(sum, ((G)c * sum + (G)1) * s)};
  else return {((G)c + P::rc(sum)) * s};
}
// tau * s for a computed s: F64 s * tau; Mixed (1/tau) / s
template <class P>
__device__ __forceinline__ Tau<P> tau_times(Tau<P> t, typename P::G s) {
  if constexpr (P::kFast) return {P::dv(t.v, s)};
  else return {s * t.v};
}
// a constant tau
template <class P>
__device__ __forceinline__ Tau<P> tau_const(double tau) {
  using G = typename P::G;
  if constexpr (P::kFast) return {(G)(1.0 / tau)};
  else return {(G)tau};
}
template <class P, bool slow = false>
__device__ __forceinline__ double rush_larsen(double y, typename P::G yinf, Tau<P> t, double dt) {
  using G = typename P::G;
  if constexpr (P::kMixed) {
    const G a = (G)dt * t.v;
    G f;
    if constexpr (slow)
      f = a * ((G)1 - a * ((G)0.5 - a * ((G)(1.0 / 6.0) - a * (G)(1.0 / 24.0))));
    else
      f = (G)1 - P::ex(-a);
    return y + (double)((yinf - (G)y) * f);
  } else if constexpr (P::kFast) {  // t.v is the rate 1/tau
    if constexpr (P::kRates) return (yinf - y) * t.v;
    const double a = dt * t.v;
    return yinf - (yinf - y) * ((slow && a < 0.1) ? exp_neg_series(a) : exp_f64(-a));
  } else {
    return rush_larsen<P, slow>(y, yinf, t.v, dt);
  }
}

// Per-instance biomarker bookkeeping (the CiPA per-beat state machine) kept in
// global memory between launches; the hot fields live in registers during a
// launch.
struct BeatRec {
  double qnet, inal_auc, ical_auc, dvmdt_repol, dvmdt_max, vm_peak, vm_valley, vm_dia, apd90,
      apd50, ca_peak, ca_valley, ca_dia, cad90, cad50;
};

// The role of a warp follows the SM sub-partition (SMSP) it was placed on
// (the warp slot modulo 4) whenever the block's four warps sit on four
// different SMSPs, so every SMSP streams one role's instructions and its
// instruction cache holds a quarter of the step's code; otherwise the warp
// index decides.
__device__ __forceinline__ int pick_role() {
  __shared__ int slot[4];
  const int w = threadIdx.x >> 5;
  unsigned wid;
  asm volatile("mov.u32 %0, %%warpid;" : "=r"(wid));
  if ((threadIdx.x & 31) == 0) slot[w] = (int)(wid & 3u);
  __syncthreads();
  const int m = (1 << slot[0]) | (1 << slot[1]) | (1 << slot[2]) | (1 << slot[3]);
  return m == 0xF ? slot[w] : w;
}

}  // namespace cep
