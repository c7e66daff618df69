/* TEST INFRASTRUCTURE ONLY: the CVODE names the reference's CiPA bench uses
 * (cipa_drug_bench.cpp:118-120,159-170,213). ref_shim/bench_shim.cpp
 * defines them: CVode advances the state by one fixed step of the oracle's
 * update scheme, so the bench's biomarker state machine can be run as
 * written on a trajectory the oracle reproduces. */
#ifndef CEP_STUB_CVODE_H
#define CEP_STUB_CVODE_H
#include <nvector/nvector_serial.h>
#define CV_BDF 2
#define CV_NEWTON 2
#define CV_NORMAL 1
#define CV_SUCCESS 0
typedef int (*CVRhsFn)(realtype t, N_Vector y, N_Vector ydot, void *user_data);
void *CVodeCreate(int lmm, int iter);
int CVodeInit(void *mem, CVRhsFn f, realtype t0, N_Vector y0);
int CVodeReInit(void *mem, realtype t0, N_Vector y0);
int CVodeSetUserData(void *mem, void *user_data);
int CVodeSStolerances(void *mem, realtype rtol, realtype atol);
int CVodeSetMaxStep(void *mem, realtype hmax);
int CVode(void *mem, realtype tout, N_Vector yout, realtype *tret, int itask);
void CVodeFree(void **mem);
#endif
