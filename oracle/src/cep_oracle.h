/*
 * TEST INFRASTRUCTURE ONLY. CPU oracle for the cardiac hot path: plain C
 * restatements of the reference cell models, their fixed-step update
 * schemes, the CiPA biomarker state machine and the FEM diffusion solve.
 * Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg load
 * this library, and only as the checker; the product never links it.
 *
 * Every function cites the reference file:line it follows (paths relative to
 * the kit-cml/2DDrugSimulation tree).
 */
#ifndef CEP_ORACLE_H
#define CEP_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- models */
enum { CEPO_ORD2011 = 0, CEPO_CIPA2017 = 1, CEPO_TT2006 = 2, CEPO_TT2004 = 3, CEPO_TOMEK2019 = 4 };

/* Largest state / parameter counts over all models. */
#define CEPO_MAX_STATES 64
#define CEPO_MAX_PARAMS 256
#define CEPO_MAX_HILL 20

/* Named per-step outputs every model fills (biomarker inputs). */
typedef struct {
  double INa, INaL, Ito, ICaL, IKr, IKs, IK1; /* channel currents (uA/uF) */
  double dVdt;                                /* RATES[V] */
} cepo_currents;

/* A model instance: constants + flags. `p` is model-specific. */
typedef struct {
  int model;
  int quirks;      /* 1: reproduce the reference's documented quirks */
  int tissue_stim; /* 0: periodic stimulus from TIME; 1: isS1 flag */
  int is_s1;       /* tissue stimulus flag */
  double p[CEPO_MAX_PARAMS];
} cepo_cell;

int cepo_n_states(int model);
/* Build constants: celltype, drug concentration, hill row (14 IC50/h pairs
 * in the reference CSV order, CiPA adds Kmax, Ku, n, halfmax, Vhalf and
 * optionally Kt at [19]), Dutta flag (ORd only), quirk mode. */
int cepo_init(cepo_cell *c, int model, double celltype, double conc, const double *hill, int n_hill,
              int is_dutta, int quirks);
void cepo_init_states(const cepo_cell *c, double *y);
/* Overrides used by the drivers (CONSTANTS[BCL], CONSTANTS[amp] *= scale). */
void cepo_set_pacing(cepo_cell *c, double bcl, double stim_start, double stim_dur, double stim_amp_scale);

/* CONSTANTS[x] *= f after init for conductance x (numbered as the
 * library's CEP_SCALE_*); -1 if the model has no such constant. */
int cepo_scale(cepo_cell *c, int g, double f);
int cepo_ord_scale(cepo_cell *c, int g, double f);
int cepo_cipa_scale(cepo_cell *c, int g, double f);
int cepo_tt06_scale(cepo_cell *c, int g, double f);
int cepo_tt04_scale(cepo_cell *c, int g, double f);
int cepo_tomek_scale(cepo_cell *c, int g, double f);

/* One fixed-step update of the reference scheme: rates at (t, y), then the
 * model's Rush-Larsen / forward-Euler update into y. `cur` (may be NULL)
 * receives the currents at (t, y). */
void cepo_step(const cepo_cell *c, double t, double dt, double *y, cepo_currents *cur);
/* Rates only (no update). dydt may be NULL. */
void cepo_rates(const cepo_cell *c, double t, const double *y, double *dydt, cepo_currents *cur);

/* ------------------------------------------------------------ biomarkers */
typedef struct {
  double qnet, inal_auc, ical_auc, dvmdt_repol, dvmdt_max, vm_peak, vm_valley, vm_dia, apd90,
      apd50, ca_peak, ca_valley, ca_dia, cad90, cad50;
} cepo_beat;

typedef struct {
  cepo_beat result;   /* selected beat (steepest repolarisation) */
  int steepest_pace;  /* pace index of `result` */
  int n_eligible;     /* eligible beats seen */
  double qnet_last;   /* qnet/1000 of the selected beat */
  int status;         /* 0 ok, 1 non-finite state */
} cepo_biomarkers;

/* Run one instance through n_pace paces at fixed dt with the biomarker
 * state machine of CEPCell_NEO/modules/cipa_drug_bench.cpp:225-330 applied
 * to paces >= first_pace (first_pace = n_pace-250 reproduces the reference;
 * first_pace = n_pace-1 is last-beat mode). ca_stride = samples of cai per
 * dt_write. Optionally records V every v_stride steps. */
int cepo_run_biomarkers(const cepo_cell *c, double *y, double dt, int n_pace, int first_pace,
                        double dt_write, double qnet_vm_threshold, cepo_biomarkers *out,
                        double *v_trace, long v_stride, long v_cap);

/* Plain fixed-step run (the reference's explicit loop), V sampled every
 * v_stride steps. t is advanced by t += dt each step. */
void cepo_run(const cepo_cell *c, double *t, double dt, long n_steps, double *y, double *v_trace,
              long v_stride);

/* Batched multi-threaded run used as the CPU baseline: n instances with
 * per-instance hill rows and concentrations, n_steps each. Returns the
 * number of threads used. */
int cepo_run_batch(int model, int n, const double *celltype, const double *conc, const double *hill,
                   int n_hill, int is_dutta, int quirks, double bcl, double dt, long n_steps,
                   double *states_out, int n_threads);

/* ------------------------------------------------------------ protocols */
/* ORd 2011: start of the current pace of the cumulative stimulus
 * (tissue_stim == 2, the CEPCell_NEO build under hrv_bench). */
void cepo_ord_set_cumm(cepo_cell *c, double cumm_bcl);

/* HRV pacing, CEPCell_NEO/modules/hrv_bench.cpp:146-343, for one cell (ORd
 * 2011, the CEPCell_NEO build: quirks 2): one pace per entry of bcls (the
 * HRV file's values and the trailing 1000 ms the bench appends), the
 * cumulative stimulus, biomarkers of the steepest of the last 250 paces.
 * Fixed steps stand for the bench's CVODE calls; every pace after the first
 * begins with the bench's zero-length call (it rewinds tcurr and tnext by dt
 * and asks for a time already reached). rec receives the printed record:
 * rec->bcl the chosen beat's BCL, *steepest its pace. */
typedef struct {
  cepo_beat beat;
  int bcl, steepest_pace;
} cepo_hrv_record;
int cepo_hrv_run(const cepo_cell *c, double *y, const double *bcls, int n_bcl, double dt, double dt_write,
                 int num_pace1, cepo_hrv_record *rec);

/* One recorded pace of a restitution run (apdr_bench.cpp:211). */
typedef struct {
  int pace, recal;
  double bcl, apd90, di, t;
} cepo_apdr_record;

/* Dynamic restitution of CEPCell_NEO/modules/apdr_bench.cpp:103-232 on the
 * fixed-step scheme; y carries the state in and out. Returns 0, or 1 when
 * V turned non-finite. *n_records = records produced (at most max_records
 * written). */
int cepo_restitution(const cepo_cell *c, double *y, const double *bcls, int n_bcl, int n_pace, double dt,
                     cepo_apdr_record *out, int max_records, int *n_records);
/* Voltage-clamp replay (CEPPatch/benchpatch.cpp:83-100). */
void cepo_clamp(const cepo_cell *c, double *y, const double *v, long n_samples, double t0, double dt,
                int current, double *out);
/* TT2004: the 2004_a build (g_Ks 0.062) after cepo_init. */
void cepo_tt04_mcell(cepo_cell *c, double conc, const double *hill);

/* -------------------------------------------------------------------- FEM */
/* Structured-grid Q1 (2D) / trilinear hex (3D) assembly of A = M/dt + K_D and
 * B = M into CSR (fem.cpp:628-661,721-752; Gauss points at +-0.57735, unit
 * weights). D is per element: either a scalar (n_d == 1) or a symmetric
 * tensor (n_d == 3 in 2D: xx,xy,yy; n_d == 6 in 3D: xx,xy,xz,yy,yz,zz). */
int cepo_fem_assemble(int dim, int nx, int ny, int nz, double h, double dt, const double *D, int n_d,
                      int *row_ptr, int *col_idx, double *a_val, double *b_val);
long cepo_fem_nnz(int dim, int nx, int ny, int nz);
/* Jacobi-PCG on CSR, zero initial guess, stop on ||r||2/||b||2 <= rtol. */
int cepo_pcg(int n, const int *row_ptr, const int *col_idx, const double *a_val, const double *b,
             double *x, double rtol, int max_iter, double *rel_res);
void cepo_spmv(int n, const int *row_ptr, const int *col_idx, const double *val, const double *x,
               double *y);
/* Same with the norm choice: precond_norm 1 = ||M^-1 r||/||M^-1 b|| (PETSc's
 * default for CG), 0 = ||r||/||b||. */
int cepo_pcg2(int n, const int *row_ptr, const int *col_idx, const double *a_val, const double *b, double *x,
              double rtol, int max_iter, int precond_norm, double *rel_res);
/* Element matrices (nn x nn, row-major) of one element of the reference's
 * kinds (0 square, 1 hex, 2 tet) with node coordinates x[nn][dim]. */
void cepo_element(int kind, const double *x, const double *D, int n_d, double dt, double *Ae, double *Be);
/* Element matrices (nn x nn, row-major) of an axis-aligned element of edge h. */
void cepo_fem_element(int dim, double h, double dt, const double *D, int n_d, double *Ae, double *Be);
/* The Godunov tissue loop on a caller's CSR operator (any mesh). */
long cepo_tissue_run_csr(int model, int n, const int *rp, const int *ci, const double *av, const double *bv, double dt,
                         long n_steps, const unsigned char *s1, double bcl, double t_crt, double dur, int n_pace,
                         double conc, const double *hill, int n_hill, double rtol, int precond_norm,
                         const double *celltype, double *V, int *iters_out, double act_thr, double *t_act);
/* P1 tetrahedral mesh: one row of the element matrices and the CSR of the
 * whole mesh (row_ptr[n_nodes+1]; col == NULL counts nnz only). */
void cepo_tet_row(const double x[4][3], const double *D, int n_d, double dt, int la, double *arow, double *brow);
long cepo_fem_assemble_tet(int n_nodes, const double *xyz, int n_elem, const int *conn, const double *D, int n_d,
                           double dt, int *row_ptr, int *col, double *a, double *b);
/* Pseudo-ECG at n_el electrodes xyz[3*k..] of a grid tissue's V
 * (Cheart::Radiate, heart.cpp:640-690). */
void cepo_pseudo_ecg(int dim, int nx, int ny, int nz, double h, const double *D, int n_d, const double *V,
                     int n_el, const double *xyz, double *phi);
/* Godunov-split tissue run on a structured grid (heart.cpp:127-165).
 * V[n] receives the final potentials, iters_out[n_steps] (or NULL) the CG
 * iterations of every step, t_act[n] (or NULL) the activation times;
 * returns the total CG iterations. */
long cepo_tissue_run(int model, int dim, int nx, int ny, int nz, double h, const double *D, int n_d, double dt,
                     long n_steps, const unsigned char *s1, double bcl, double t_crt, double dur, int n_pace,
                     double conc, const double *hill, int n_hill, double rtol, int precond_norm,
                     const double *celltype, double *V, int *iters_out, double act_thr, double *t_act);
/* The same with the S1-S2 reset (s2_kind 1) or ectopic (2) protocol. */
long cepo_tissue_run_s2(int model, int dim, int nx, int ny, int nz, double h, const double *D, int n_d, double dt,
                        long n_steps, const unsigned char *s1, double bcl, double t_crt, double dur, int n_pace,
                        double conc, const double *hill, int n_hill, double rtol, int precond_norm,
                        const double *celltype, double *V, int *iters_out, double act_thr, double *t_act,
                        int s2_kind, int target, double thr, const unsigned char *region, double ecto_dur);

#ifdef __cplusplus
}
#endif
#endif
