/* TEST INFRASTRUCTURE ONLY: see cvode.h. */
#ifndef CEP_STUB_CVODE_DENSE_H
#define CEP_STUB_CVODE_DENSE_H
#include <cvode/cvode.h>
int CVDense(void *mem, long n);
#endif
