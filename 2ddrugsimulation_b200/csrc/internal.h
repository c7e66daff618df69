// Library-internal entry points shared between the translation units (not
// part of the C ABI).
#pragma once
#include "../../include/cep_b200.h"

// S1-S2 / ectopic protocol state of a tissue (Cheart::apply_s2 and
// Cheart::apply_ectopic, heart.cpp:452-501), kept in device memory and
// updated on the device before every ionic step.
struct CepProto {
  int kind;        // CEP_S2_NONE, CEP_S2_RESET or CEP_S2_ECTOPIC
  int target;      // monitored node
  double thr;      // mV: depolarised above, repolarised below
  double dur;      // ectopic stimulus length, ms
  int depol, repol, fired;
  int reset_now;   // reset the S2 region in this step
  int ecto_on;     // ectopic region stimulated in this step
  double t_fire;
};

#ifdef __cplusplus
extern "C" {
#endif

// One Godunov ionic step of a tissue at tissue time t: every node advances
// by the batch's dt with the stimulus flag isS1 = mask[i] while
// iia*bcl + t_crt < t < iia*bcl + t_crt + dur and iia = (int)(t/bcl) < n_pace
// (heart.cpp:309-323). d_mask is a device array of n bytes. With a device
// protocol state (may be NULL) the S1 flag is off once the protocol has
// fired, and nodes of d_mask2 are stimulated while its ectopic flag is on.
// Asynchronous.
int cep_internal_batch_tissue_step(cep_batch_t b, const unsigned char *d_mask, double t, double bcl, double t_crt,
                                   double dur, int n_pace, const struct CepProto *proto,
                                   const unsigned char *d_mask2);
// Tissue clock: every instance at t = 0 with no protocol end and biomarkers
// off; the fixed step is dt.
int cep_internal_batch_tissue_begin(cep_batch_t b, double dt);
// Device pointer of the membrane-potential row (n doubles) and the stream.
double *cep_internal_batch_v(cep_batch_t b);
void *cep_internal_batch_stream(cep_batch_t b);
// Records an error message for cep_last_error and returns code.
int cep_internal_set_fail(int code, const char *msg);

#ifdef __cplusplus
}
#endif
