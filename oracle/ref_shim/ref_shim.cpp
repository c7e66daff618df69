/*
 * TEST INFRASTRUCTURE ONLY -- never linked into the product library.
 *
 * C-ABI wrapper around one unmodified reference cell-model class, compiled
 * directly from the reference sources (see oracle/Makefile). It exposes the
 * reference object's public arrays and its computeRates/solveAnalytical calls
 * so the tests can pin the CPU restatement (oracle/src) against the
 * reference itself, and so bench.py can time the reference CPU path.
 *
 * One translation unit per model: the build passes
 *   -DREF_HEADER="..."  the reference model header
 *   -DREF_CLASS=...     the reference model class
 *   -DREF_INIT_KIND=N   which initConsts overload the model offers
 *        1: initConsts(celltype, conc, ic50[14], is_dutta)   (ORd 2011,
 *           DrugSimulation/cellmodels/Ohara_Rudy_2011.cpp:722)
 *        2: initConsts(celltype, conc, hill[])               (CiPA-ORd,
 *           CEPCell_NEO/cellmodels/ohara_rudy_cipa_v1_2017.cpp:1515; Tomek
 *           CEPCell_NEO/cellmodels/Tomek_model.cpp:1149; TT2004b
 *           CEPCell_NEO/cellmodels/tentusscher_noble_noble_panfilov_2004_b.cpp:361)
 *        3: initConsts()                                    (TT2006,
 *           CEPCell_NEO/cellmodels/ten_tusscher_model_2006_IK1Ko_epi_units.cpp:196)
 *        4: like 2 but the class stores arrays inline (Cellmodel base)
 *   -DREF_INLINE_ARRAYS  the class derives from Cellmodel (arrays inline)
 *   -DREF_NEO_HRV        adds ref_set_hrv (the CEPCell_NEO ORd's HRV stimulus)
 */
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include REF_HEADER
#ifdef REF_NEO_HRV
#include "globals.hpp"
#endif

/* The reference's cell models print through mpi_printf
 * (DrugSimulation/modules/glob_funct.hpp:16); the oracle silences it. */
void mpi_printf(unsigned short, const char *, ...) {}
void mpi_fprintf(unsigned short, FILE *, const char *, ...) {}

extern "C" {

void *ref_new(void) { return new REF_CLASS(); }
void ref_free(void *h) { delete static_cast<REF_CLASS *>(h); }

int ref_sizes(void *h, int *n_states, int *n_consts, int *n_alg) {
  REF_CLASS *c = static_cast<REF_CLASS *>(h);
  *n_states = (int)c->states_size;
  *n_consts = (int)c->constants_size;
  *n_alg = (int)c->algebraic_size;
  return 0;
}

/* celltype, conc and a hill/ic50 row; is_dutta only for kind 1. */
void ref_init(void *h, double celltype, double conc, double *hill, int is_dutta) {
  REF_CLASS *c = static_cast<REF_CLASS *>(h);
#if REF_INIT_KIND == 1
  c->initConsts(celltype, conc, hill, is_dutta != 0);
#elif REF_INIT_KIND == 2
  (void)is_dutta;
  c->initConsts(celltype, conc, hill);
#else
  (void)celltype; (void)conc; (void)hill; (void)is_dutta;
  c->initConsts();
#endif
}

double *ref_states(void *h) { return static_cast<REF_CLASS *>(h)->STATES; }
double *ref_consts(void *h) { return static_cast<REF_CLASS *>(h)->CONSTANTS; }
double *ref_rates(void *h) { return static_cast<REF_CLASS *>(h)->RATES; }
double *ref_alg(void *h) { return static_cast<REF_CLASS *>(h)->ALGEBRAIC; }
void ref_set_s1(void *h, int on) { static_cast<REF_CLASS *>(h)->isS1 = (on != 0); }
void ref_set_ectopic(void *h, int on) { static_cast<REF_CLASS *>(h)->isEctopic = (on != 0); }

void ref_compute_rates(void *h, double t) {
  REF_CLASS *c = static_cast<REF_CLASS *>(h);
  c->computeRates(t, c->CONSTANTS, c->RATES, c->STATES, c->ALGEBRAIC);
}
void ref_solve(void *h, double dt) { static_cast<REF_CLASS *>(h)->solveAnalytical(dt); }

/* The reference's explicit loop (CEPCell_HACKATHON/modules/
 * cipa_drug_explicit_bench.cpp:119-127): computeRates(tcurr); solve(dt);
 * tcurr += dt. Records STATES[0] after every `stride` steps into v_out
 * (may be NULL). Returns the final tcurr through *t. */
void ref_run(void *h, double *t, double dt, long n_steps, double *v_out, long stride) {
  REF_CLASS *c = static_cast<REF_CLASS *>(h);
  double tc = *t;
  long k = 0;
  for (long i = 0; i < n_steps; ++i) {
    c->computeRates(tc, c->CONSTANTS, c->RATES, c->STATES, c->ALGEBRAIC);
    c->solveAnalytical(dt);
    tc += dt;
    if (v_out && stride > 0 && ((i + 1) % stride) == 0) v_out[k++] = c->STATES[0];
  }
  *t = tc;
}

#ifdef REF_NEO_HRV
/* The CEPCell_NEO ORd switches its stimulus to the cumulative-BCL window
 * when glob_var::is_hrv is set (CEPCell_NEO/cellmodels/Ohara_Rudy_2011.cpp:
 * 694-695); CONSTANTS[cumm_BCL] (141) is set through ref_consts. */
void ref_set_hrv(int on) { glob_var::is_hrv = (on != 0); }
#endif

}  // extern "C"
