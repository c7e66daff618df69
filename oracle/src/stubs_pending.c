/* TEST INFRASTRUCTURE ONLY. Placeholders for models whose restatement is
 * not written yet; each reports failure. */
#include "cep_oracle.h"
#define STUB(pfx)                                                                          \
  int cepo_##pfx##_init(cepo_cell *c, double a, double b, const double *h, int d, int q) { \
    (void)c; (void)a; (void)b; (void)h; (void)d; (void)q; return -1; }                  \
  void cepo_##pfx##_set_pacing(cepo_cell *c, double a, double b, double d, double e) {     \
    (void)c; (void)a; (void)b; (void)d; (void)e; }                                        \
  void cepo_##pfx##_pacing(const cepo_cell *c, double *a, double *b) { (void)c; *a = 0; *b = 0; } \
  void cepo_##pfx##_step(const cepo_cell *c, double t, double dt, double *y, cepo_currents *k) { \
    (void)c; (void)t; (void)dt; (void)y; (void)k; }                                       \
  void cepo_##pfx##_rates(const cepo_cell *c, double t, const double *y, double *r, cepo_currents *k) { \
    (void)c; (void)t; (void)y; (void)r; (void)k; }
STUB(tomek)
void cepo_tomek_init_states(const cepo_cell *c, double *y) { (void)c; (void)y; }
