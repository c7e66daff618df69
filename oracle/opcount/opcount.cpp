// TEST/MEASUREMENT INFRASTRUCTURE ONLY. Counts the algorithmic operations of
// one fixed-step cell update by compiling the oracle's restatement with an
// operation-counting scalar in place of `double`. A value is "constant" when
// it derives only from literals and instance parameters; an operation whose
// operands are all constant is foldable at initialisation and is not
// counted. Output: per-step counts averaged over whole beats.
//
//   make -C oracle opcount && oracle/_build/opcount <model> <beats> <bcl>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>

struct Counts {
  long add = 0, mul = 0, div = 0, ex = 0, lg = 0, pw = 0, sq = 0, fl = 0, cmp = 0;
};
static Counts g_cnt;
static bool g_on = false;

struct od {
  double v;
  bool k;  // true: depends on constants only
  od() = default;
  od(double x) : v(x), k(true) {}
  od(int x) : v(x), k(true) {}
  od(long x) : v((double)x), k(true) {}
  explicit operator double() const { return v; }
  explicit operator int() const { return (int)v; }
};
static inline od mk(double v, bool k) { od r; r.v = v; r.k = k; return r; }
#define BIN(opch, field)                                                                   \
  static inline od operator opch(od a, od b) {                                             \
    if (g_on && !(a.k && b.k)) g_cnt.field++;                                              \
    return mk(a.v opch b.v, a.k && b.k);                                                   \
  }                                                                                        \
  static inline od operator opch(od a, double b) { return a opch od(b); }                  \
  static inline od operator opch(double a, od b) { return od(a) opch b; }
BIN(+, add) BIN(-, add) BIN(*, mul) BIN(/, div)
#undef BIN
static inline od operator-(od a) { return mk(-a.v, a.k); }
static inline od &operator+=(od &a, od b) { a = a + b; return a; }
static inline od &operator-=(od &a, od b) { a = a - b; return a; }
static inline od &operator*=(od &a, od b) { a = a * b; return a; }
static inline od &operator/=(od &a, od b) { a = a / b; return a; }
#define CMP(opch)                                                                      \
  static inline bool operator opch(od a, od b) {                                       \
    if (g_on && !(a.k && b.k)) g_cnt.cmp++;                                            \
    return a.v opch b.v;                                                               \
  }                                                                                    \
  static inline bool operator opch(od a, double b) { return a opch od(b); }            \
  static inline bool operator opch(double a, od b) { return od(a) opch b; }
CMP(<) CMP(>) CMP(<=) CMP(>=) CMP(==) CMP(!=)
#undef CMP
#define UN(name, field)                                                      \
  static inline od name(od a) {                                              \
    if (g_on && !a.k) g_cnt.field++;                                         \
    return mk(std::name(a.v), a.k);                                          \
  }
UN(exp, ex) UN(log, lg) UN(sqrt, sq) UN(floor, fl) UN(ceil, fl) UN(fabs, cmp)
#undef UN
static inline od pow(od a, od b) {
  if (g_on && !(a.k && b.k)) {
    // integral exponents are products on the GPU (x^2 = 1 mul, ..., x^8 = 3)
    const double e = b.v;
    if (b.k && (e == 2.0 || e == 3.0 || e == 4.0 || e == 8.0 || e == -1.0)) {
      g_cnt.mul += e == 2.0 ? 1 : e == 3.0 ? 2 : e == 4.0 ? 2 : e == 8.0 ? 3 : 0;
      if (e == -1.0) g_cnt.div++;
    } else if (b.k && e == 0.5) {
      g_cnt.sq++;
    } else {
      g_cnt.pw++;
    }
  }
  return mk(std::pow(a.v, b.v), a.k && b.k);
}
static inline od pow(od a, double b) { return pow(a, od(b)); }
static inline od copysign(od a, od b) { return mk(std::copysign(a.v, b.v), a.k && b.k); }

#define double od
#define _Static_assert static_assert
#define memset(p, c, n) ::std::memset((void *)(p), c, n)
#include "../src/cep_oracle.h"
#include "../src/ord2011.c"
#define V V_cipa_
#undef V
namespace cipa_ns {
#include "../src/cipa2017.c"
}
namespace tt06_ns {
#include "../src/tt2006.c"
}
namespace tt04_ns {
#include "../src/tt2004.c"
}
namespace tomek_ns {
#include "../src/tomek2019.c"
}
#undef double

int main(int argc, char **argv) {
  const char *model = argc > 1 ? argv[1] : "cipa2017";
  const int beats = argc > 2 ? atoi(argv[2]) : 1;
  const double bcl = argc > 3 ? atof(argv[3]) : 1000.0;
  const double dt = 0.005;
  cepo_cell c;
  od y[64];
  od hill[20];
  for (int k = 0; k < 20; ++k) hill[k] = od(0.0);
  const long n = (long)(beats * bcl / dt);
  void (*step)(const cepo_cell *, od, od, od *, cepo_currents *) = nullptr;
  if (!strcmp(model, "ord2011")) {
    cepo_ord_init(&c, od(0.0), od(0.0), hill, 0, 1);
    cepo_ord_set_pacing(&c, od(bcl), od(-1.0), od(-1.0), od(1.0));
    cepo_ord_init_states(y);
    step = cepo_ord_step;
  } else if (!strcmp(model, "cipa2017")) {
    hill[14] = 10; hill[15] = 0.001; hill[16] = 0.9; hill[17] = 1000; hill[18] = -50; hill[19] = 3.5e-5;
    cipa_ns::cepo_cipa_init(&c, od(0.0), od(1.0), hill, 0, 1);
    cipa_ns::cepo_cipa_set_pacing(&c, od(bcl), od(-1.0), od(-1.0), od(1.0));
    cipa_ns::cepo_cipa_init_states(&c, y);
    step = cipa_ns::cepo_cipa_step;
  } else if (!strcmp(model, "tt2006")) {  // epicardial, as the tissue sheets
    tt06_ns::cepo_tt06_init(&c, od(2.0), od(0.0), hill, 0, 1);
    tt06_ns::cepo_tt06_set_pacing(&c, od(bcl), od(-1.0), od(-1.0), od(1.0));
    tt06_ns::cepo_tt06_init_states(y);
    step = tt06_ns::cepo_tt06_step;
  } else if (!strcmp(model, "tt2004")) {
    tt04_ns::cepo_tt04_init(&c, od(2.0), od(0.0), hill, 0, 1);
    tt04_ns::cepo_tt04_set_pacing(&c, od(bcl), od(-1.0), od(-1.0), od(1.0));
    tt04_ns::cepo_tt04_init_states(y);
    step = tt04_ns::cepo_tt04_step;
  } else if (!strcmp(model, "tomek2019")) {
    tomek_ns::cepo_tomek_init(&c, od(0.0), od(0.0), hill, 0, 1);
    tomek_ns::cepo_tomek_set_pacing(&c, od(bcl), od(-1.0), od(-1.0), od(1.0));
    tomek_ns::cepo_tomek_init_states(&c, y);
    step = tomek_ns::cepo_tomek_step;
  } else {
    std::fprintf(stderr, "unknown model %s\n", model);
    return 2;
  }
  c.tissue_stim = 0;
  for (int k = 0; k < 64; ++k) y[k].k = false;  // states are variables
  od t = od(0.0);
  t.k = false;
  for (long s = 0; s < n; ++s) {
    g_on = true;
    step(&c, t, od(dt), y, nullptr);
    g_on = false;
    t = mk(t.v + dt, false);
  }
  const double f = 1.0 / (double)n;
  std::printf("{\"model\": \"%s\", \"steps\": %ld, \"add\": %.2f, \"mul\": %.2f, \"div\": %.2f, \"exp\": %.2f, "
              "\"log\": %.2f, \"pow\": %.2f, \"sqrt\": %.2f, \"floor\": %.2f, \"cmp\": %.2f, \"V_end\": %.6f}\n",
              model, n, g_cnt.add * f, g_cnt.mul * f, g_cnt.div * f, g_cnt.ex * f, g_cnt.lg * f, g_cnt.pw * f,
              g_cnt.sq * f, g_cnt.fl * f, g_cnt.cmp * f, y[0].v);
  return 0;
}
