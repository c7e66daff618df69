/* TEST INFRASTRUCTURE ONLY: the SUNDIALS serial-vector names the
 * reference's CiPA bench uses (CEPCell_NEO/modules/commons.hpp,
 * cipa_drug_bench.cpp), as a plain wrapper of a caller's array. SUNDIALS is
 * not in the reference tree as source; ref_shim/bench_shim.cpp defines
 * these functions. */
#ifndef CEP_STUB_NVECTOR_SERIAL_H
#define CEP_STUB_NVECTOR_SERIAL_H
typedef double realtype;
struct cep_nvector {
  long length;
  realtype *data;
};
typedef struct cep_nvector *N_Vector;
N_Vector N_VMake_Serial(long length, realtype *data);
realtype *N_VGetArrayPointer_Serial(N_Vector v);
void N_VDestroy(N_Vector v);
void N_VDestroy_Serial(N_Vector v);
#endif
