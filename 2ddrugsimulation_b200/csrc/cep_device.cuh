// Shared device-side definitions for the ionic-model kernels.
//
// Two precision policies drive every model template:
//   F64   - plain FP64 path: every quantity in double, libm-equivalent exp/log
//           (CUDA's double exp/log, <= 1 ulp), reference expression order.
//   Mixed - gates, rate constants and channel currents in FP32 with SFU
//           exp/log (ex2.approx / lg2.approx) and approximate division; the
//           membrane voltage, the ionic concentrations, CaMKII and every
//           accumulation stay FP64.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace cep {

struct F64 {
  using G = double;
  static constexpr bool kMixed = false;
  __device__ __forceinline__ static double ex(double x) { return ::exp(x); }
  __device__ __forceinline__ static double lg(double x) { return ::log(x); }
  __device__ __forceinline__ static double dv(double a, double b) { return a / b; }
  __device__ __forceinline__ static double rc(double x) { return 1.0 / x; }
  __device__ __forceinline__ static double pw(double x, double y) { return ::pow(x, y); }
  __device__ __forceinline__ static double sq(double x) { return ::sqrt(x); }
};

struct Mixed {
  using G = float;
  static constexpr bool kMixed = true;
  __device__ __forceinline__ static float ex(float x) { return __expf(x); }
  __device__ __forceinline__ static float lg(float x) { return __logf(x); }
  __device__ __forceinline__ static float dv(float a, float b) { return __fdividef(a, b); }
  __device__ __forceinline__ static float rc(float x) { return __fdividef(1.0f, x); }
  __device__ __forceinline__ static float pw(float x, float y) { return __powf(x, y); }
  __device__ __forceinline__ static float sq(float x) { return sqrtf(x); }
};

// x^2, x^3, x^4, x^8 by repeated products (the reference calls pow() with
// integral exponents; products differ from a correctly rounded pow by at
// most an ulp).
template <class T> __device__ __forceinline__ T p2(T x) { return x * x; }
template <class T> __device__ __forceinline__ T p3(T x) { return x * x * x; }
template <class T> __device__ __forceinline__ T p4(T x) { T y = x * x; return y * y; }
template <class T> __device__ __forceinline__ T p8(T x) { T y = x * x; y = y * y; return y * y; }

// x / (e^x - 1), the Goldman-Hodgkin-Katz factor, evaluated without the
// cancellation the direct form suffers for |x| -> 0 (series below 1e-3).
__device__ __forceinline__ float ghk_factor(float x) {
  if (fabsf(x) < 1e-3f) return 1.0f - 0.5f * x + x * x * (1.0f / 12.0f);
  return __fdividef(x, __expf(x) - 1.0f);
}

// Rush-Larsen update y_inf - (y_inf - y) * exp(-dt/tau).
template <class P>
__device__ __forceinline__ typename P::G rush_larsen(typename P::G y, typename P::G yinf,
                                                     typename P::G tau, typename P::G dt) {
  return yinf - (yinf - y) * P::ex(P::dv(-dt, tau));
}

// Per-instance biomarker bookkeeping (the CiPA per-beat state machine) kept in
// global memory between launches; the hot fields live in registers during a
// launch.
struct BeatRec {
  double qnet, inal_auc, ical_auc, dvmdt_repol, dvmdt_max, vm_peak, vm_valley, vm_dia, apd90,
      apd50, ca_peak, ca_valley, ca_dia, cad90, cad50;
};

}  // namespace cep
