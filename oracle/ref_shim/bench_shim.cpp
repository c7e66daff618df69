/*
 * TEST INFRASTRUCTURE ONLY -- never linked into the product library.
 *
 * Runs the reference's CiPA drug bench (CEPCell_NEO/modules/
 * cipa_drug_bench.cpp, compiled unmodified with its commons.cpp) on a
 * trajectory the oracle can reproduce, so that the bench's per-step
 * biomarker state machine (:225-330) and its records (:352-380) pin the
 * oracle's restatement of that machine (oracle/src/cell.c).
 *
 *  - The bench constructs `new Ohara_Rudy_2011()` against the CEPCell_NEO
 *    header. This shim defines that class's members (declared in
 *    CEPCell_NEO/cellmodels/Ohara_Rudy_2011.hpp) over the oracle's ORd 2011
 *    restatement (intended forms, no quirks): initConsts builds an oracle
 *    cell, computeRates fills RATES and the seven channel currents at the
 *    NEO enum indices from the oracle's rates.
 *  - SUNDIALS is present only as prebuilt libraries, so CVODE is replaced
 *    by the stand-ins of ref_shim/sundials: CVode(tout) advances the state
 *    by one fixed step of the oracle's scheme (cepo_step) from the previous
 *    output time. MPI is one process.
 *
 * The cell model is therefore the oracle's own; what the comparison pins is
 * the bench's sampling, pace bookkeeping, steepest-beat choice, Ca and APD
 * crossing rules and qNet / qInward arithmetic.
 */
#include <unistd.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>

#include "../modules/cipa_drug_bench.hpp"
#include "../modules/commons.hpp"
#include "../modules/hrv_bench.hpp"
#include "../modules/globals.hpp"
#include "Ohara_Rudy_2011.hpp"
#include "cep_oracle.h"
#include <cvode/cvode.h>
#include <cvode/cvode_dense.h>
#include <mpi.h>

namespace {
struct OracleCell {
  cepo_cell c;
  double bcl = 1000.0, amp = -80.0, gna = 75.0;
};
std::map<const patch_clamp *, OracleCell> g_cells;
// hrv_bench runs the CEPCell_NEO build (oracle quirk mode 2) with its
// cumulative stimulus (the oracle's tissue_stim 2)
bool g_hrv = false;

// a caller's CONSTANTS writes (cipa_drug_bench.cpp:146-148) into the oracle cell
void sync_consts(const patch_clamp *p, const double *C) {
  OracleCell &o = g_cells[p];
  if (C[BCL] != o.bcl || C[amp] != o.amp) {
    cepo_set_pacing(&o.c, C[BCL], -1.0, -1.0, C[amp] / o.amp);
    o.bcl = C[BCL];
    o.amp = C[amp];
  }
  if (C[GNa] != o.gna) {
    cepo_scale(&o.c, 0, C[GNa] / o.gna);
    o.gna = C[GNa];
  }
  if (g_hrv) cepo_ord_set_cumm(&o.c, C[cumm_BCL]);
}

struct CvMem {
  void *user = nullptr;
  double t = 0.0;
};
}  // namespace

// ------------------------------------------------ the bench's cell class
Ohara_Rudy_2011::Ohara_Rudy_2011() {
  algebraic_size = 198;
  constants_size = 142;
  states_size = 41;
  ALGEBRAIC = new double[algebraic_size]();
  CONSTANTS = new double[constants_size]();
  RATES = new double[states_size]();
  STATES = new double[states_size]();
  isS1 = false;
  isEctopic = false;
}
Ohara_Rudy_2011::~Ohara_Rudy_2011() {
  g_cells.erase(this);
  delete[] ALGEBRAIC;
  delete[] CONSTANTS;
  delete[] RATES;
  delete[] STATES;
}
void Ohara_Rudy_2011::___applyDutta() {}
void Ohara_Rudy_2011::___initConsts() {}
void Ohara_Rudy_2011::initConsts() { initConsts(0.0, 0.0, nullptr, false); }
void Ohara_Rudy_2011::initConsts(double type) { initConsts(type, 0.0, nullptr, false); }
void Ohara_Rudy_2011::initConsts(double type, bool is_dutta) { initConsts(type, 0.0, nullptr, is_dutta); }
void Ohara_Rudy_2011::initConsts(double type, double D, double *hill, bool is_dutta) {
  OracleCell o;
  cepo_init(&o.c, CEPO_ORD2011, type, D, hill, hill ? 14 : 0, is_dutta ? 1 : 0, g_hrv ? 2 : 0);
  if (g_hrv) o.c.tissue_stim = 2;
  cepo_init_states(&o.c, STATES);
  g_cells[this] = o;
  // the pacing the bench reads back (stimulus at 10 ms for 0.5 ms: the
  // oracle's ORd defaults, as initConsts sets them, Ohara_Rudy_2011.cpp)
  CONSTANTS[BCL] = o.bcl;
  CONSTANTS[amp] = o.amp;
  CONSTANTS[GNa] = o.gna;
  CONSTANTS[stim_start] = 10.0;
  CONSTANTS[duration] = 0.5;
  CONSTANTS[cumm_BCL] = 0.0;
}
void Ohara_Rudy_2011::computeRates(double TIME, double *C, double *R, double *S, double *A) {
  sync_consts(this, C);
  cepo_currents cur;
  cepo_rates(&g_cells[this].c, TIME, S, R, &cur);
  A[INa] = cur.INa; A[INaL] = cur.INaL; A[Ito] = cur.Ito; A[ICaL] = cur.ICaL;
  A[IKr] = cur.IKr; A[IKs] = cur.IKs; A[IK1] = cur.IK1;
}

// ------------------------------------------------ SUNDIALS / MPI stand-ins
N_Vector N_VMake_Serial(long length, realtype *data) { return new cep_nvector{length, data}; }
realtype *N_VGetArrayPointer_Serial(N_Vector v) { return v->data; }
void N_VDestroy(N_Vector v) { delete v; }
void N_VDestroy_Serial(N_Vector v) { delete v; }
void *CVodeCreate(int, int) { return new CvMem(); }
int CVodeInit(void *mem, CVRhsFn, realtype t0, N_Vector) {
  static_cast<CvMem *>(mem)->t = t0;
  return CV_SUCCESS;
}
int CVodeReInit(void *mem, realtype t0, N_Vector) {
  static_cast<CvMem *>(mem)->t = t0;
  return CV_SUCCESS;
}
int CVodeSetUserData(void *mem, void *user) {
  static_cast<CvMem *>(mem)->user = user;
  return CV_SUCCESS;
}
int CVodeSStolerances(void *, realtype, realtype) { return CV_SUCCESS; }
int CVodeSetMaxStep(void *, realtype) { return CV_SUCCESS; }
int CVDense(void *, long) { return CV_SUCCESS; }
int CVode(void *mem, realtype tout, N_Vector y, realtype *tret, int) {
  CvMem *m = static_cast<CvMem *>(mem);
  const patch_clamp *p = static_cast<const patch_clamp *>(m->user);
  sync_consts(p, p->CONSTANTS);
  // a time already reached (hrv_bench.cpp:185-192 rewinds tnext by dt) is no
  // step: the state stays as it is
  if (tout > m->t) {
    cepo_step(&g_cells[p].c, m->t, tout - m->t, y->data, nullptr);
    m->t = tout;
  }
  *tret = tout;
  return CV_SUCCESS;
}
void CVodeFree(void **mem) {
  delete static_cast<CvMem *>(*mem);
  *mem = nullptr;
}
int MPI_Barrier(MPI_Comm) { return 0; }
double MPI_Wtime(void) { return 0.0; }

// ------------------------------------------------ driver
extern "C" int ref_cipa_bench(const char *workdir, const char *hill_file, const char *concs, const char *drug,
                              double celltype, double bcl, double dt, double dt_write, int num_pace) {
  // the bench frees its parameter block when it ends (cipa_drug_bench.cpp:458)
  param_t &p = *static_cast<param_t *>(std::calloc(1, sizeof(param_t)));
  set_default_values(&p);
  p.celltype = celltype;
  p.bcl_init = bcl;
  p.dt = dt;
  p.dt_write = dt_write;
  p.num_pace1 = num_pace;
  // graph output on: with it off the bench writes the per-pace repolarisation
  // slopes through a FILE* it never opened (fp_maxdvdt_repol,
  // cipa_drug_bench.cpp:47,176-186,258) and crashes at the first eligible
  // beat
  p.is_print_graph = 1;
  p.is_using_output = 0;
  p.stim_amp = 1.0;
  p.gna_scale = 1.0;
  std::snprintf(p.hill_file, sizeof(p.hill_file), "%s", hill_file);
  std::snprintf(p.concs, sizeof(p.concs), "%s", concs);
  std::snprintf(p.drug_name, sizeof(p.drug_name), "%s", drug);
  mympi::rank = 0;
  mympi::size = 1;
  char cwd[4096];
  if (!getcwd(cwd, sizeof(cwd)) || chdir(workdir) != 0) return 1;
  cipa_drug_bench(0, nullptr, &p, true);  // writes result/result_<drug>_<time>.zip
  return chdir(cwd) == 0 ? 0 : 2;
}

// The reference's HRV bench (hrv_bench.cpp) over the same cell: one pace per
// line of the HRV file, results in result/<conc>/ (not zipped).
extern "C" int ref_hrv_bench(const char *workdir, const char *hill_file, const char *hrv_file, const char *concs,
                             const char *drug, double celltype, double dt, double dt_write, int num_pace) {
  param_t &p = *static_cast<param_t *>(std::calloc(1, sizeof(param_t)));
  set_default_values(&p);
  p.celltype = celltype;
  p.dt = dt;
  p.dt_write = dt_write;
  p.num_pace1 = num_pace;
  p.is_print_graph = 0;
  p.stim_amp = 1.0;
  std::snprintf(p.hill_file, sizeof(p.hill_file), "%s", hill_file);
  std::snprintf(p.hrv_files, sizeof(p.hrv_files), "%s", hrv_file);
  std::snprintf(p.concs, sizeof(p.concs), "%s", concs);
  std::snprintf(p.drug_name, sizeof(p.drug_name), "%s", drug);
  mympi::rank = 0;
  mympi::size = 1;
  glob_var::is_hrv = true;
  g_hrv = true;
  char cwd[4096];
  if (!getcwd(cwd, sizeof(cwd)) || chdir(workdir) != 0) return 1;
  hrv_bench(0, nullptr, &p);
  g_hrv = false;
  glob_var::is_hrv = false;
  return chdir(cwd) == 0 ? 0 : 2;
}
