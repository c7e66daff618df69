/*
 * cep_b200 -- B200-native cardiac drug-screening hot path: batched ionic-model
 * stepping with Hill-equation drug block and on-device biomarkers, and the
 * monodomain FEM diffusion solve.
 *
 * Plain C ABI: opaque handles, host pointers and sizes, int status codes. No
 * CUDA or torch types appear in the signatures (device pointers are passed
 * as void*). Every entry point returns CEP_OK (0) or a CEP_ERR_* code;
 * cep_last_error() gives the message of the calling thread's last failure.
 *
 * Threading: a handle is bound to one CUDA stream and must not be used from
 * two host threads at once. Handles are independent of each other.
 *
 * Each entry point names the reference interface it replaces (paths are
 * within the kit-cml/2DDrugSimulation tree).
 */
#ifndef CEP_B200_H
#define CEP_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status */
#define CEP_OK 0
#define CEP_ERR_ARG 1           /* invalid argument (null, size, range)     */
#define CEP_ERR_OOM 2           /* device allocation failed                 */
#define CEP_ERR_CUDA 3          /* CUDA runtime error                       */
#define CEP_ERR_NOT_CONVERGED 4 /* iterative solve hit max_iter             */
#define CEP_ERR_TIMEOUT 5       /* a bounded device wait ran out            */
#define CEP_ERR_NONFINITE 6     /* a state became NaN/Inf (per instance)    */
#define CEP_ERR_UNSUPPORTED 7   /* model/precision combination not built   */
#define CEP_ERR_STATE 8         /* call out of order (e.g. run before init) */
#define CEP_ERR_NO_DEVICE 9     /* no CUDA device visible                   */

/* per-instance status words (cep_batch_get_status) */
#define CEP_INST_RUNNING 0
#define CEP_INST_DONE 1     /* reached the end of its protocol */
#define CEP_INST_NONFINITE 2 /* state left the finite range; frozen */
#define CEP_INST_IDLE 3      /* slot released (cep_batch_release_range) */

/* ----------------------------------------------------------------- models */
#define CEP_MODEL_ORD2011 0   /* DrugSimulation/cellmodels/Ohara_Rudy_2011.cpp, 41 states */
#define CEP_MODEL_CIPA2017 1  /* CEPCell_NEO/cellmodels/ohara_rudy_cipa_v1_2017.cpp, 49 states */
#define CEP_MODEL_TT2006 2    /* CEPCell_NEO/cellmodels/ten_tusscher_model_2006_IK1Ko_epi_units.cpp, 19 states */
#define CEP_MODEL_TT2004 3    /* CEPCell_NEO/cellmodels/tentusscher_noble_noble_panfilov_2004_b.cpp, 17 states */
#define CEP_MODEL_TOMEK2019 4 /* CEPCell_NEO/cellmodels/Tomek_model.cpp, 43 states */

#define CEP_PREC_FP64 0  /* everything in FP64                                  */
#define CEP_PREC_MIXED 1 /* FP32 gates/rates/currents, FP64 V, ions, CaMKII     */

/* init flags */
#define CEP_FLAG_DUTTA 1u  /* Dutta et al. 2017 conductance scaling (ORd)          */
#define CEP_FLAG_QUIRKS 2u /* reproduce the reference's documented quirks exactly  */
#define CEP_FLAG_TT04_MCELL 4u /* TT2004: the 2004_a build (g_Ks 0.062, M cell) instead of
                                  2004_b (g_Ks 0.245): tentusscher_noble_noble_panfilov_2004_a.cpp:265,
                                  chosen by celltype 0 in apdr_bench.cpp:77-84 */
#define CEP_FLAG_NEO_ORD 8u /* ORd 2011: the CEPCell_NEO build driven by the HRV bench
                               (CEPCell_NEO/cellmodels/Ohara_Rudy_2011.cpp:456-520):
                               celltype honoured, Dutta on the intended constants and
                               the Hill block after PCap/PCaNa/PCaK were derived, so
                               those stay unscaled. Not with CEP_FLAG_QUIRKS. */

/* state array layouts for set/get */
#define CEP_LAYOUT_SOA 0 /* states[k * n + i] (k = state index, i = instance) */
#define CEP_LAYOUT_AOS 1 /* states[i * n_states + k]                          */

/* Width of one Hill row: 14 IC50/h pairs in the reference CSV column order
 * (ICaL, IK1, IKs, INa, INaL, Ito, hERG: CEP5Cell/bin/drugs/<drug>/
 * IC50_samples.csv:1), then the CiPA dynamic-hERG set Kmax, Ku, n,
 * halfmax, Vhalf (CEPCell_NEO/cellmodels/ohara_rudy_cipa_v1_2017.cpp:1534-1538)
 * and Kt. IC50 or h <= 1e-13 means "no block" (the reference reads NA as 0). */
#define CEP_HILL_WIDTH 20

/* One beat's biomarkers: the fields of cipa_t (CEPCell_NEO/modules/
 * commons.hpp:18-36) as the CiPA bench prints them (cipa_drug_bench.cpp:
 * 352-379). qnet is in the reference's printed unit (integral / 1000). */
typedef struct {
  double qnet, inal_auc, ical_auc;
  double dvmdt_repol, dvmdt_max, vm_peak, vm_valley, vm_dia, apd90, apd50, apd_tri;
  double ca_peak, ca_valley, ca_dia, cad90, cad50, cad_tri;
  int32_t steepest_pace; /* pace index the result was taken from          */
  int32_t n_eligible;    /* eligible beats evaluated                       */
  int32_t status;        /* CEP_INST_*                                     */
  int32_t reserved;
} cep_biomarkers_t;

typedef struct cep_batch *cep_batch_t;

/* Library identity. */
const char *cep_version(void);
const char *cep_last_error(void);
/* Number of visible CUDA devices (0 on a host without GPUs). */
int cep_device_count(void);

/* Create a batch of n instances of one model on the current CUDA device,
 * bound to `stream` (a cudaStream_t, NULL = the legacy default stream).
 * Replaces `new Ohara_Rudy_2011()` / `new ohara_rudy_cipa_v1_2017()` per
 * instance (cellmodel.hpp:4-36, patch_clamp.hpp:4-26). */
int cep_batch_create(int model, int n, int precision, void *stream, cep_batch_t *out);
int cep_batch_destroy(cep_batch_t b);
int cep_batch_size(cep_batch_t b, int *n, int *n_states);
/* Threads per block of the run kernel (32, 64, 96 or 128); the default
 * spreads small populations over every SM. Used by the autotuner. */
int cep_batch_set_block(cep_batch_t b, int threads_per_block);
/* Kernel form: one thread per cell; 4 warps per 32 cells each evaluating
 * one group of channels; or 2 warps per 32 cells with two groups each (ORd
 * family only). Defaults for populations below ~1.5 waves of the GPU: FP64
 * the 4 roles; mixed the 4 roles up to one 32-cell group per SM and the
 * pairs above; larger populations one thread per cell. */
#define CEP_KERNEL_CELL 0
#define CEP_KERNEL_ROLES 1
#define CEP_KERNEL_PAIRS 2 /* 2 warps per 32 cells, two channel groups each */
int cep_batch_set_kernel(cep_batch_t b, int variant);
/* Launch-shape autotuner (no counterpart in the reference, which runs one
 * cell per object): times one run of n_steps steps (default 400) in each
 * kernel form and block size on this batch's own instances and keeps the
 * fastest. Every array a run writes (states, clocks, status, biomarker
 * records, Ca ring) is saved first and restored after every trial, so the
 * batch continues exactly where it was. Blocking; needs room for one copy
 * of those arrays. The chosen form and block are returned if the pointers
 * are not NULL. */
int cep_batch_autotune(cep_batch_t b, long n_steps, int *variant, int *block);

/* initConsts for every instance and the model's initial STATES.
 * celltype[n] (NULL = 0, endo), conc[n] (drug concentration, same unit as
 * IC50), hill[n * hill_stride] (NULL = no drug), flags CEP_FLAG_*.
 * Replaces Ohara_Rudy_2011::initConsts(type, conc, ic50, is_dutta)
 * (Ohara_Rudy_2011.cpp:722-738) and ohara_rudy_cipa_v1_2017::
 * initConsts(type, conc, hill) (ohara_rudy_cipa_v1_2017.cpp:1515-1539).
 * The Hill scaling runs on the device. */
int cep_batch_init(cep_batch_t b, const double *celltype, const double *conc, const double *hill,
                   int hill_stride, unsigned flags);

/* Pacing overrides applied after init: CONSTANTS[BCL] = bcl,
 * CONSTANTS[stim_start], CONSTANTS[duration], CONSTANTS[amp] *= amp_scale
 * (cipa_drug_bench.cpp:146-147). Negative stim_start / stim_dur keep the
 * model defaults. */
int cep_batch_set_pacing(cep_batch_t b, double bcl, double stim_start, double stim_dur, double amp_scale);

/* Per-instance conductance scaling applied after init, the reference's
 * CONSTANTS[x] *= scale at its call sites: the deck's G*_Scale keys
 * (CONSTANTS[GNa] *= gna_scale, cipa_drug_bench.cpp:148, heart.cpp:222;
 * the TT benches' g_Ks .. g_pK, anm_bench_custom.cpp:62-71) and the
 * population-of-models sweeps (population_tn2006.cpp:72-101: ten scale
 * factors per instance). factor[n] multiplies the named conductance of
 * every instance; like the reference, a derived constant computed inside
 * initConsts from it (ORd's PCap from PCa) is left as it is.
 * CEP_ERR_UNSUPPORTED for a conductance the model does not have as a
 * parameter (ORd's background currents are fixed constants). */
enum {
  CEP_SCALE_GNA = 0, CEP_SCALE_GNAL, CEP_SCALE_GTO, CEP_SCALE_GCAL, CEP_SCALE_GKR, CEP_SCALE_GKS,
  CEP_SCALE_GK1, CEP_SCALE_GBNA, CEP_SCALE_GBCA, CEP_SCALE_GPCA, CEP_SCALE_GPK, CEP_SCALE_GKB,
  CEP_SCALE_GNCX, CEP_SCALE_PNAK, CEP_SCALE_COUNT
};
int cep_batch_scale(cep_batch_t b, int conductance, const double *factor);
/* The same conductance of every instance read or written as values[n]
 * (the instance's CONSTANTS entry after init, scaling and Hill block).
 * cep::Cellmodel mirrors these at the reference's CONSTANTS indices, so a
 * caller's CONSTANTS[GNa] *= gna_scale (heart.cpp:222) reaches the device
 * unchanged. Blocking. */
int cep_batch_get_conductance(cep_batch_t b, int conductance, double *values);
int cep_batch_set_conductance(cep_batch_t b, int conductance, const double *values);

/* Protocol of the run: fixed step dt (ms), n_pace paces at the instance's
 * BCL, biomarkers evaluated on paces >= first_pace (first_pace = n_pace-250
 * reproduces cipa_drug_bench.cpp:296; n_pace-1 is last-beat mode; -1 turns
 * biomarkers off), Ca sampled every dt_write ms for CaD50/90, qNet summed
 * while V > qnet_vm_threshold (-1e300: always, as cipa_drug_bench.cpp:225;
 * -88: as heart.cpp:369). Resets every instance's clock to t = 0. */
int cep_batch_set_protocol(cep_batch_t b, double dt, int n_pace, int first_pace, double dt_write,
                           double qnet_vm_threshold);

/* Advance every unfinished instance by up to n_steps fixed steps of the
 * reference scheme (computeRates then solveAnalytical, t += dt:
 * cipa_drug_explicit_bench.cpp:119-127) with the biomarker state machine
 * fused. Asynchronous on the batch's stream. */
int cep_batch_run(cep_batch_t b, long n_steps);
/* One fixed step of every instance from time t: the reference's loop body
 * computeRates(t, ...); solveAnalytical(dt) (cipa_drug_explicit_bench.cpp:
 * 119-127; heart.cpp:330-360 per node). stim_mode -1: the model's periodic
 * single-cell stimulus at t; 0/1: the tissue flag isS1 for every instance.
 * No biomarker bookkeeping and no clock update (the caller owns t).
 * Asynchronous on the batch's stream. */
int cep_batch_step(cep_batch_t b, double t, double dt, int stim_mode);
/* Run to the end of the protocol (blocking). */
int cep_batch_run_to_end(cep_batch_t b, long steps_per_launch);

/* Host <-> device state transfer (blocking). layout CEP_LAYOUT_*. */
int cep_batch_set_states(cep_batch_t b, const double *states, int layout);
int cep_batch_get_states(cep_batch_t b, double *states, int layout);
/* Device pointer of the SoA state block ([n_states][ld] doubles). */
int cep_batch_device_states(cep_batch_t b, void **dev_ptr, long *ld);

int cep_batch_get_biomarkers(cep_batch_t b, cep_biomarkers_t *out /* [n] */);
int cep_batch_get_status(cep_batch_t b, int32_t *status /* [n] */);
/* Checkpoint / resume of a whole batch mid-protocol (the reference writes
 * node states to output.<rank> and resumes with iopt = 1, heart.cpp:141,
 * 595-616, 943-963; this also keeps the clocks, schedules, parameters and
 * the biomarker state machine with its Ca ring, so a resumed run ends
 * bit-identical to an uninterrupted one). The blob is self-describing and
 * restores into a batch created with the same model, size and precision.
 * Both calls are blocking. */
int cep_batch_checkpoint_size(cep_batch_t b, size_t *bytes);
int cep_batch_checkpoint(cep_batch_t b, void *buf, size_t bytes);
int cep_batch_restore(cep_batch_t b, const void *buf, size_t bytes);
/* Current step count and time of instance i. */
int cep_batch_get_clock(cep_batch_t b, int i, long *step, double *t);
int cep_batch_sync(cep_batch_t b);

/* Rates at the current state without advancing it (computeRates,
 * Ohara_Rudy_2011.cpp:742): dVdt[n] and the seven channel currents
 * currents[7*n] (INa, INaL, Ito, ICaL, IKr, IKs, IK1; SoA). */
int cep_batch_rates(cep_batch_t b, double t, double *dvdt, double *currents);
/* The whole RATES vector at the current state, as computeRates fills it for
 * an ODE solver (the reference's CVODE right-hand side rhs_fn,
 * CEPCell_NEO/modules/commons.cpp:26-35; ORd computeRates
 * Ohara_Rudy_2011.cpp:742-989): rates[n * n_states] (AoS, the STATES order),
 * a gate's (y_inf - y)/tau and every other state's forward-Euler
 * derivative, in FP64. ORd 2011, CiPA-ORd and ToR-ORd; the ten Tusscher
 * models (stepped with their own solveAnalytical) return
 * CEP_ERR_UNSUPPORTED. Blocking. */
int cep_batch_rates_all(cep_batch_t b, double t, double *rates);

/* ------------------------------------------------------- whole jobs */
/* One screening job: the CiPA bench loop over every sample and
 * concentration (CEPCell_NEO/modules/cipa_drug_bench.cpp:128-380:
 * initConsts(celltype, conc, hill, is_dutta), CONSTANTS[BCL] = bcl,
 * CONSTANTS[amp] *= stim_amp, CONSTANTS[GNa] *= gna_scale (here any of the
 * CEP_SCALE_* conductances per instance), optional initial states, n_pace
 * paces, biomarkers from the steepest evaluated beat) as
 * one population on the device. precision CEP_PREC_MIXED with a finite
 * refine_above_vm keeps the mixed path's accuracy bar for every instance:
 * after screen_paces mixed paces, the instances whose membrane potential
 * at the pace boundary is above refine_above_vm (drug-depolarised cells
 * that do not repolarise, whose APD90 FP32 gates cannot hold) run from
 * their initial state in FP64 on a second stream concurrently with the
 * mixed population, and any instance whose evaluated record still shows a
 * diastolic Vm above it, an APD90 above 0.9 BCL or an intermittent rhythm
 * (0 < n_eligible < the evaluated paces: the edge of 2:1 block, whose
 * regime FP32 rounding can change) runs again in FP64
 * afterwards (refined[i] = 1 concurrent, 2 afterwards). refine_above_vm =
 * NaN (or CEP_PREC_FP64) runs the single precision alone. No counterpart
 * in the reference beyond the loop it replaces. Blocking. */
typedef struct {
  int model, n;
  const double *celltype; /* [n] or NULL (endo) */
  const double *conc;     /* [n] or NULL */
  const double *hill;     /* [n * hill_stride] or NULL */
  int hill_stride;
  unsigned flags;         /* CEP_FLAG_* */
  double bcl, amp_scale;
  const double *scale;       /* [n * CEP_SCALE_COUNT] factors (cep_batch_scale) or NULL */
  const double *states_init; /* one state vector for every instance, or NULL */
  double dt, dt_write;
  int n_pace, first_pace;
  int precision;
  double refine_above_vm; /* mV; NaN: no refinement */
  int screen_paces;       /* >= 1 */
  long steps_per_launch;  /* <= 0: 20000 */
} cep_population_job_t;
/* out[n] receives the records; refined[n] (may be NULL) 0 for a mixed
 * record, 1 for an FP64 record of a screened instance, 2 for one re-run
 * after the mixed run. */
int cep_population_run(const cep_population_job_t *job, cep_biomarkers_t *out, int *refined);
/* The rule of step 3 above on n mixed records, for callers that run their
 * own batches: mask[i] = 1 when record i shows a diastolic Vm not below
 * refine_above_vm (a NaN Vm included), an APD90 above 0.9 bcl, or an
 * intermittent rhythm (0 < n_eligible < evaluated, evaluated = the paces
 * from first_pace on); else 0. Host only, no device work. */
int cep_population_late_mask(const cep_biomarkers_t *recs, int n, double refine_above_vm, double bcl, int evaluated,
                             int *mask);

/* ------------------------------------------------- protocol variants */
/* One pace of a dynamic (S1-S1) restitution run, as apdr_bench.cpp:211
 * writes it ("all_pace bcl apd90 t_di tcurr"); recal = 1 when the pace's
 * windowed Vm peak was below 10 mV and the APD came from the search over the
 * pace's whole Vm trace (:172-191). */
typedef struct {
  int32_t pace;  /* running pace number over all BCLs (all_pace)        */
  int32_t recal; /* 1: the recalibration search set the APD              */
  double bcl;    /* ms                                                   */
  double apd90;  /* ms                                                   */
  double di;     /* diastolic interval: next stimulus - repolarisation   */
  double t;      /* segment clock at the end of the pace (tcurr)         */
} cep_apdr_record_t;

/* Dynamic restitution of every instance (apdr_bench.cpp:103-232, the CVODE
 * integration replaced by the fixed-step scheme): for each bcl[s] in order,
 * CONSTANTS[BCL] = bcl[s], the segment clock restarts at 0 and the cell
 * state carries over; iout = 1 .. (int)(n_pace*bcl/dt) + 1 steps; at every
 * pace boundary (iout % (int)(bcl/dt) == 0) the pace's APD90 (90 %
 * repolarisation from the peak in (start+4, start+56) ms against the
 * previous boundary's Vm) is closed, and paces after the first two of each
 * BCL are recorded. out[n * max_records] (instance-major); *n_records
 * receives the records per instance (the same for every instance; at most
 * max_records are written). The run keeps each instance's Vm over the
 * current pace in device memory (max over s of (int)(bcl[s]/dt) doubles
 * per instance) for the recalibration search. Blocking.
 * apdr_bcls() in the Python package builds the reference's BCL list
 * (bcl_init down to bcl_end, decrement 10 once bcl <= 300). */
int cep_batch_restitution(cep_batch_t b, const double *bcl, int n_bcl, int n_pace, double dt,
                          long steps_per_launch, cep_apdr_record_t *out, int max_records, int *n_records);

/* Voltage-clamp replay (CEPPatch/benchpatch.cpp:83-100): before step k the
 * membrane potential of every instance is set to v[k]; the step runs the
 * model from t0 + k*dt (t += dt) with its periodic stimulus; out[k * n + i]
 * receives channel current `current` of instance i at that step (0 INa,
 * 1 INaL, 2 Ito, 3 ICaL, 4 IKr, 5 IKs, 6 IK1: the order of
 * cep_batch_rates). The instances' states advance; the batch clock is not
 * touched. Blocking. */
int cep_batch_clamp(cep_batch_t b, const double *v, long n_samples, double t0, double dt, int current,
                    double *out);

/* The HRV bench's result for one instance: the beat it prints (qnet in the
 * printed unit, integral / 1000; steepest_pace = the pace it came from;
 * status CEP_INST_DONE or CEP_INST_NONFINITE) and that beat's BCL as the
 * bench prints it, (int)BCL. */
typedef struct {
  cep_biomarkers_t beat;
  int32_t bcl;
  int32_t reserved;
} cep_hrv_record_t;

/* Heart-rate-variability pacing (CEPCell_NEO/modules/hrv_bench.cpp:
 * 146-343, the CVODE integration replaced by the fixed-step scheme):
 * pace p lasts bcls[p] ms (the bench's interval file with 1000 ms
 * appended), the stimulus starts stim_start after the cumulative start of
 * the pace (CONSTANTS[cumm_BCL], Ohara_Rudy_2011.cpp:694-695), the clock
 * carries over between paces with the bench's one-step rewind at each
 * pace start (a zero-length first call), and the CiPA biomarkers of the
 * last 250 paces are evaluated (none when n_bcl < 250, as the bench's
 * size_t arithmetic gives); the beat with the steepest repolarisation is
 * kept, the beat of pace num_pace1 - 250 replaces it once, and APD90 <
 * APD50 reports APD90 = BCL. ORd 2011 batches only (the model the bench
 * drives; CEP_FLAG_NEO_ORD at init gives its build). The instances' states
 * advance. out[n]. steps_per_launch <= 0 picks 20,000. Blocking. */
int cep_batch_hrv(cep_batch_t b, const double *bcls, int n_bcl, double dt, double dt_write, int num_pace1,
                  long steps_per_launch, cep_hrv_record_t *out);

/* ---------------------------------------------------- instance ranges */
/* Heterogeneous batches: a batch used as a pool of slots whose ranges hold
 * different jobs at different points of their protocols (the serving
 * loop). No counterpart in the reference, which runs one job per process.
 *
 * reserve_biomarkers: fixes the batch-wide step dt, the Ca sampling
 * interval and the qNet threshold, reserves the biomarker records and a Ca
 * ring of max_samples_per_beat (= BCL/dt_write of the longest beat), and
 * releases every slot. Instances of a running job are never touched by
 * calls on other ranges. */
int cep_batch_reserve_biomarkers(cep_batch_t b, int max_samples_per_beat, double dt, double dt_write,
                                 double qnet_vm_threshold);
/* initConsts for instances [first, first+count); inputs indexed from 0. */
int cep_batch_init_range(cep_batch_t b, int first, int count, const double *celltype, const double *conc,
                         const double *hill, int hill_stride, unsigned flags);
int cep_batch_set_pacing_range(cep_batch_t b, int first, int count, double bcl, double stim_start,
                               double stim_dur, double amp_scale);
/* Start the range's protocol: n_pace paces at each instance's BCL with
 * biomarkers from first_pace (-1: off); clocks reset to t = 0 and the
 * instances marked running. */
int cep_batch_start_range(cep_batch_t b, int first, int count, int n_pace, int first_pace);
/* Mark the range idle: run launches skip it. */
int cep_batch_release_range(cep_batch_t b, int first, int count);
int cep_batch_get_biomarkers_range(cep_batch_t b, int first, int count, cep_biomarkers_t *out);

/* --------------------------------------------------------------- serving */
/* A screening-job server with continuous batching (no counterpart in the
 * reference). One pool of `capacity` slots stays resident in HBM; each
 * job (a list of instances: samples x concentrations with their Hill rows)
 * is admitted into a free slot range as soon as one fits, runs inside the
 * same launches as every other admitted job, and is collected and released
 * when all its instances finish. A job's biomarkers are bit-identical alone
 * or in any mix. capacity <= 0 sizes the pool to hbm_fraction of the free
 * device memory (the admission budget); max_bcl bounds the BCL of jobs that
 * want biomarkers (it sizes the Ca ring). One scheduler thread per server. */
typedef struct cep_server *cep_server_t;

#define CEP_JOB_QUEUED 0
#define CEP_JOB_RUNNING 1
#define CEP_JOB_DONE 2
#define CEP_JOB_FAILED 3
#define CEP_JOB_CANCELLED 4

typedef struct {
  int n;                  /* instances                                    */
  const double *celltype; /* [n] or NULL (endo)                           */
  const double *conc;     /* [n]                                          */
  const double *hill;     /* [n * hill_stride] or NULL                    */
  int hill_stride;
  double bcl;             /* ms                                           */
  int n_pace, first_pace; /* protocol as cep_batch_set_protocol           */
  unsigned flags;         /* CEP_FLAG_*                                   */
} cep_job_t;

typedef struct {
  double queue_ms;   /* submit -> admission                  */
  double run_ms;     /* admission -> completion              */
  double latency_ms; /* submit -> completion                 */
  double cell_steps; /* instance-steps of the job            */
} cep_job_times_t;

typedef struct {
  int capacity, queued, running, slots_used;
  long long completed, launches;
  double cell_steps; /* instance-steps of completed jobs      */
  double busy_ms;    /* time inside launches + status reads  */
  double wall_ms;    /* since start                          */
} cep_serve_stats_t;

int cep_serve_start(int model, int precision, int capacity, double dt, double dt_write, double max_bcl,
                    long steps_per_launch, double hbm_fraction, void *stream, cep_server_t *out);
int cep_serve_submit(cep_server_t s, const cep_job_t *job, uint64_t *id);
int cep_serve_poll(cep_server_t s, uint64_t id, int *state);
/* Block until the job is done (timeout_s <= 0: no limit). */
int cep_serve_wait(cep_server_t s, uint64_t id, double timeout_s);
/* out[job n] biomarkers (may be NULL) and timings (may be NULL). */
int cep_serve_result(cep_server_t s, uint64_t id, cep_biomarkers_t *out, cep_job_times_t *times);
/* Forget a finished job (frees its host-side record). */
int cep_serve_release(cep_server_t s, uint64_t id);
/* Cancel a job: a queued one leaves at once; a running one leaves between
 * two launches (its slots return to the pool, a patch's device memory is
 * freed) and never blocks the others. Its state becomes CEP_JOB_CANCELLED
 * and cep_serve_wait returns CEP_ERR_STATE for it. */
int cep_serve_cancel(cep_server_t s, uint64_t id);
int cep_serve_stats(cep_server_t s, cep_serve_stats_t *st);

/* A 2D TT2006 tissue patch as a screening job (an nx x ny sheet of Q1 nodes
 * with a corner S1 block, the drug as one Hill row on every node). Admitted
 * while the server's HBM budget has room for it, then stepped with every
 * other running patch as one tissue group (one batched PCG launch per step)
 * on a stream of its own, overlapping the population pool's launches. Its
 * V and activation times are those of running the patch alone (to the
 * PCG's tolerance). No counterpart in the reference (one Cheart per run,
 * heart.cpp). */
typedef struct {
  int nx, ny;           /* nodes                                       */
  double h;             /* node spacing, cm                            */
  double D;             /* isotropic conductivity, cm^2/ms             */
  double dt;            /* ionic and diffusion step, ms                */
  double duration;      /* simulated time, ms                          */
  double conc;          /* drug concentration                          */
  const double *hill;   /* [14] Hill row (TT2006 uses IKr: hill[12..13]) or NULL */
  double bcl;           /* S1 period, ms (S1 at t = k*bcl for 1 ms)     */
  int stim_nx, stim_ny; /* S1 corner block, nodes                      */
  double rtol;          /* PCG tolerance (<= 0: 1e-8)                  */
} cep_tissue_job_t;
int cep_serve_submit_tissue(cep_server_t s, const cep_tissue_job_t *job, uint64_t *id);
/* Final V and activation times ([nx*ny] each, -1: never activated; either
 * may be NULL) and timings of a finished tissue job. */
int cep_serve_tissue_result(cep_server_t s, uint64_t id, double *v, double *t_act, cep_job_times_t *times);
/* Stop the scheduler (queued and running jobs fail), free the pool. */
int cep_serve_stop(cep_server_t s);

/* qInward of a drug run against its control: 0.5*(INaL_auc_drug/
 * INaL_auc_ctrl + ICaL_auc_drug/ICaL_auc_ctrl) (cipa_drug_bench.cpp:376). */
double cep_qinward(const cep_biomarkers_t *control, const cep_biomarkers_t *drug);

/* ------------------------------------------------------ monodomain FEM */
/* The diffusion operator of one tissue: A = M/dt + D K and B = M, with the
 * implicit step A V = B V* / dt solved by Jacobi-preconditioned CG from a
 * zero initial guess. Replaces Cfem::assemble_Amat_Bmat (fem.cpp:721-763),
 * Cfem::set_amat_bmat (fem.cpp:628-661) and Cfem::solve_Bmat
 * (fem.cpp:705-718) with PETSc KSPCG + PCJACOBI (fem.cpp:753-760). */
typedef struct cep_fem *cep_fem_t;

#define CEP_FEM_AUTO (-1) /* time every format this operator has (40-iteration solves), keep the fastest */
#define CEP_FEM_CSR 0
#define CEP_FEM_ELL 1     /* column-major ELL, padded to the widest row */
#define CEP_FEM_STENCIL 2 /* grid operators: 9/27 fixed slots, implicit columns */
#define CEP_FEM_CLASSED 3 /* grid operators: a class index per row, coefficients per class */

/* Structured grid of nx*ny (dim 2, Q1 quadrilaterals) or nx*ny*nz (dim 3,
 * trilinear hexahedra) nodes at spacing h (cm), node id i + nx*(j + ny*k),
 * the reference's "square" / hex meshes (mesh.cpp, fem.cpp:231-271,398-478).
 * D holds n_d values per element, element id ex + (nx-1)*(ey + (ny-1)*ez):
 * n_d = 1 is the reference's scalar DE (fem.cpp:656); n_d = 3 (2D: xx, xy,
 * yy) or 6 (3D: xx, xy, xz, yy, yz, zz) is a conductivity tensor. Assembly
 * runs on the device. stream as in cep_batch_create. */
int cep_fem_create_grid(int dim, int nx, int ny, int nz, double h, double dt, const double *D, int n_d,
                        int format, void *stream, cep_fem_t *out);
/* An unstructured mesh of linear tetrahedra (the reference's "tet" meshes,
 * mesh.cpp:59-186; Gauss points fem.cpp:209-229, shape functions
 * fem.cpp:342-373, element matrices fem.cpp:628-661): xyz[n_nodes*3] (cm),
 * conn[n_elem*4] (0-based nodes), D[n_elem*n_d] with n_d 1 (scalar, the
 * reference's DE) or 6 (xx, xy, xz, yy, yz, zz). Assembled on the device,
 * one thread per row summing its incident elements in ascending order; CSR
 * or ELL (or CEP_FEM_AUTO between them). No pseudo-ECG on these operators. */
int cep_fem_create_tet(int n_nodes, const double *xyz, int n_elem, const int *conn, const double *D, int n_d,
                       double dt, int format, void *stream, cep_fem_t *out);
/* An operator assembled by the caller (any mesh), CSR with sorted columns. */
int cep_fem_create_csr(int n, const int *row_ptr, const int *col_idx, const double *a_val, const double *b_val,
                       double dt, int format, void *stream, cep_fem_t *out);
int cep_fem_destroy(cep_fem_t f);
int cep_fem_info(cep_fem_t f, int *n, long *nnz, int *format, int *ell_width);
int cep_fem_set_format(cep_fem_t f, int format);
/* Host copy of the assembled CSR (row_ptr[n+1], col_idx/a_val/b_val[nnz]). */
int cep_fem_get_csr(cep_fem_t f, int *row_ptr, int *col_idx, double *a_val, double *b_val);
/* Stopping rule ||r|| <= rtol ||b|| after at most max_iter iterations, in the
 * preconditioned norm ||D^-1 r|| (precond_norm = 1, PETSc's default for CG)
 * or the plain 2-norm. Defaults: rtol 1e-5 (PETSc's default; the reference
 * sets none), max_iter 10000, preconditioned norm. max_iter is at most
 * CEP_FEM_MAX_ITER (the grid barrier counts arrivals in 31 bits). */
#define CEP_FEM_MAX_ITER 1000000
int cep_fem_set_solver(cep_fem_t f, double rtol, int max_iter, int precond_norm);
/* y = A x (which = 0) or B x (which = 1); host vectors of n doubles. */
int cep_fem_spmv(cep_fem_t f, int which, const double *x, double *y);
/* One implicit diffusion step on a host vector: in V*, out V (blocking). */
int cep_fem_solve(cep_fem_t f, double *v, int *iters, double *rel_res);
/* The same on a device vector of n doubles, asynchronous on the stream. */
int cep_fem_solve_device(cep_fem_t f, void *d_v);
/* Solver counters (blocking): iterations of the last solve (negative when
 * it hit max_iter), iterations and solves summed, solves that hit max_iter,
 * relative residual of the last solve. CEP_ERR_TIMEOUT if a device barrier
 * ran out of its spin limit. */
int cep_fem_stats(cep_fem_t f, int *last_iters, long *total_iters, long *solves, int *not_converged,
                  double *last_res);

/* Test hook of the bounded device waits (no counterpart in the reference):
 * every grid barrier of the PCG kernels on the current device gives up
 * after spin_limit polls (0 restores the default of ~1-2 s) and block 0
 * sleeps block0_delay_ns (at most 0.1 s) before its first barrier. With a
 * short limit and a delay, the other blocks' waits run out: the solve ends
 * early, every block leaves, and the blocking calls report CEP_ERR_TIMEOUT;
 * the context stays usable. Reset with (0, 0). */
int cep_fem_set_wait_test(long spin_limit, unsigned block0_delay_ns);

/* Allocation-free solve. No counterpart in the reference. One implicit
 * diffusion step A V = B V / dt, Jacobi-PCG from a zero guess with the
 * default stopping rule (preconditioned norm), for a CSR operator the
 * caller keeps in device memory (d_row_ptr[n+1], d_col_idx/d_a_val/
 * d_b_val[nnz], sorted columns), in place on the device vector d_v[n].
 * Nothing is allocated or freed: the solver's work vectors live in a fixed
 * device scratch area of the library sized for CEP_NOALLOC_MAX_ROWS rows
 * (larger n is rejected with CEP_ERR_ARG). The first call on a device
 * resolves that area and must come before any stream capture. Calls that
 * overlap in time on one device (two streams or two host threads) share
 * the scratch and race: serialise them. The scratch address is resolved
 * once per device and assumes the device is never reset (cudaDeviceReset)
 * while the library is loaded. Asynchronous on `stream` unless iters_out is
 * non-null, in which case the call waits and stores the iteration count and
 * reports CEP_ERR_NOT_CONVERGED past max_iter, CEP_ERR_TIMEOUT when a device
 * barrier ran out of its spin limit, and CEP_ERR_ARG for a row without a
 * usable (present, nonzero, finite) diagonal entry. The asynchronous form
 * reports none of these: the next call clears the status words, and d_v may
 * hold a partial solve. A row without a usable diagonal is preconditioned
 * with 1 in both forms. */
#define CEP_NOALLOC_MAX_ROWS 262144
int cep_fem_solve_csr_noalloc(int n, const void *d_row_ptr, const void *d_col_idx, const void *d_a_val,
                              const void *d_b_val, double dt, double rtol, int max_iter, void *d_v, void *stream,
                              int *iters_out);

/* ---------------------------------------------------------------- tissue */
/* Godunov-split monodomain tissue: per step every node's ionic update (the
 * batch, one instance per node, tissue stimulus flag isS1) then the implicit
 * diffusion solve on the V row, in place on the device (Cheart::processing,
 * heart.cpp:127-165; Cheart::cellular_reaction, heart.cpp:274-430). The
 * batch must be initialised, have as many instances as the operator has
 * rows, share its stream, and dt must equal the operator's. Creating the
 * tissue resets the batch's clock to t = 0 and turns its biomarkers off. */
typedef struct cep_tissue *cep_tissue_t;
int cep_tissue_create(cep_batch_t cells, cep_fem_t fem, double dt, cep_tissue_t *out);
int cep_tissue_destroy(cep_tissue_t t);
/* S1 nodes (mask[n], nonzero = stimulated) are driven while
 * iia*bcl + t_crt < t < iia*bcl + t_crt + dur for pace iia = (int)(t/bcl)
 * < n_pace (the "square" mesh rule, heart.cpp:309-323). */
int cep_tissue_set_stimulus(cep_tissue_t t, const unsigned char *s1_mask, double bcl, double t_crt, double dur,
                            int n_pace);
/* Activation time of a node = the first step end at which V >= threshold
 * (default -30 mV); -1 until then. No counterpart in the reference. */
int cep_tissue_set_activation_threshold(cep_tissue_t t, double vm_threshold);
/* Set the tissue clock (ms), e.g. to the time of an output.<rank> snapshot
 * whose node states were loaded with cep_batch_set_states: the resume of
 * heart.cpp:595-616 (iopt = 1). Blocking. */
int cep_tissue_set_clock(cep_tissue_t t, double time);
/* Advance n_steps Godunov steps (asynchronous). */
int cep_tissue_run(cep_tissue_t t, long n_steps);
int cep_tissue_sync(cep_tissue_t t);
int cep_tissue_get_v(cep_tissue_t t, double *v);
int cep_tissue_get_activation(cep_tissue_t t, double *t_act);
int cep_tissue_stats(cep_tissue_t t, double *time, long *steps, long *cg_iters, int *not_converged);
/* Pseudo-ECG (Cheart::Radiate, heart.cpp:640-690, and its callers at
 * heart.cpp:560-576): after every `every`-th step the tissue records, for
 * each of n_el electrodes at xyz[3*k..] (cm; node (i, j, k) of the grid sits
 * at (i h, j h, k h)), phi = w sum_elements sum_gauss (D grad V) . (c - x)
 * detJ / |c - x|^3, c the element centroid, w = 1/6 as the reference; at
 * most max_records records are kept on the device. The reference's
 * uninitialised Gauss counter and its accumulator that is never reset
 * between calls are not reproduced. Grid operators only
 * (CEP_ERR_UNSUPPORTED otherwise); n_el = 0 turns it off. */
int cep_tissue_set_electrodes(cep_tissue_t t, int n_el, const double *xyz, long every, long max_records);
/* Copy the records so far (phi[n_records][n_el]; phi may be NULL). */
int cep_tissue_get_ecg(cep_tissue_t t, double *phi, long *n_records);
/* S1-S2 protocols of the reference (Cheart::apply_s2 / apply_ectopic,
 * heart.cpp:452-501, armed at heart.cpp:322-323), evaluated on the device
 * before every ionic step of the last S1 pace ((int)(t/bcl) == n_pace - 1 of
 * cep_tissue_set_stimulus): once the monitored node has risen above
 * vm_threshold and fallen back below it, the protocol fires once and the S1
 * stimulus stays off. CEP_S2_RESET (the reference uses -45 mV) sets every
 * node of region[n] back to the states it had when this call was made (call
 * it before running: the initial states); CEP_S2_ECTOPIC (-75 mV) drives
 * the region with the S1 stimulus current for ectopic_dur ms (isEctopic),
 * switched off, as in the reference, only while still in that pace.
 * CEP_S2_NONE disarms. */
#define CEP_S2_NONE 0
#define CEP_S2_RESET 1
#define CEP_S2_ECTOPIC 2
int cep_tissue_set_s2(cep_tissue_t t, int kind, int target_node, double vm_threshold, const unsigned char *region,
                      double ectopic_dur);

/* A group of tissues stepped together: each keeps its own cells, operator,
 * stimulus and solver state, but their diffusion solves share one
 * cooperative launch per step (grid blocks split in proportion to rows), so
 * the CG barrier latency is paid once for the whole group. The tissues must
 * share one stream and sparse format (and grid dimension); each keeps its
 * own time and dt; at most one tissue per SM. Results are those of stepping
 * each tissue alone (to the solver's tolerance: the PCG's block partition
 * depends on the group). Replaces running one Cheart (heart.cpp) per
 * concentration or request. */
typedef struct cep_tissue_group *cep_tissue_group_t;
int cep_tissue_group_create(const cep_tissue_t *tissues, int count, cep_tissue_group_t *out);
int cep_tissue_group_run(cep_tissue_group_t g, long n_steps);
int cep_tissue_group_destroy(cep_tissue_group_t g);
/* Per-phase device time of the steps run while timing is on: CUDA events
 * on the group's stream before the ionic launches, before the diffusion
 * launch and after it, each step. set_timing resets the totals; timing()
 * waits for the recorded steps and returns the totals since then. No
 * counterpart in the reference (its timing is host wall clock around the
 * whole run, heart.cpp). */
int cep_tissue_group_set_timing(cep_tissue_group_t g, int on);
int cep_tissue_group_timing(cep_tissue_group_t g, double *ionic_ms, double *diffusion_ms, long *steps);

/* ---------------------------------------------------------- slab parts */
/* A structured-grid tissue split into parts that each own a contiguous
 * range of planes (the last axis: y in 2D, z in 3D), one part per GPU: the
 * reference's row distribution of A, B and V (MatCreateMPIAIJ with
 * PETSC_DECIDE, fem.cpp:667-670; the ghost exchange and dot-product
 * reductions inside MatMult / KSPSolve, fem.cpp:705-718). The part holds its
 * rows of A and B (bit-identical to the same rows of cep_fem_create_grid's
 * operator) and the split Jacobi-PCG; moving the boundary planes between
 * neighbouring parts and gathering the parts' partial sums is the
 * caller's (NCCL or peer copies across GPUs; plain device buffers for
 * several parts on one GPU). No V is gathered: each part's cells need only
 * their own rows.
 *
 * split: planes [first, first + planes) of part `part`, the first
 * n_planes % n_parts parts one plane longer (PETSc's PETSC_DECIDE rule).
 * create_grid: arguments as cep_fem_create_grid with the whole grid's D
 * (host); the part keeps the elements its rows touch. info: global index
 * of the first owned row, owned rows (whole planes), rows per plane, and
 * whether a lower / upper neighbour exists. get_csr: the owned rows with
 * global column indices. */
typedef struct cep_part *cep_part_t;
int cep_part_split(int n_planes, int n_parts, int part, int *first_plane, int *planes);
int cep_part_create_grid(int dim, int nx, int ny, int nz, double h, double dt, const double *D, int n_d, int part,
                         int n_parts, void *stream, cep_part_t *out);
int cep_part_destroy(cep_part_t p);
int cep_part_info(cep_part_t p, long *row0, long *n_own, long *plane, int *has_lo, int *has_hi);
int cep_part_get_csr(cep_part_t p, int *row_ptr, int *col_idx, double *a_val, double *b_val);
/* rtol, max_iter and the norm as cep_fem_set_solver (same defaults). */
int cep_part_set_solver(cep_part_t p, double rtol, int max_iter, int precond_norm);
/* One implicit diffusion step A V = B V / dt split across the parts (all
 * asynchronous on the part's stream; device pointers; a plane is `plane`
 * doubles; partial buffers are 2 doubles per part, `all` the n_parts
 * parts' partials in part order):
 *   pack(d_v, lo, hi)          the first / last owned plane of V into lo / hi
 *                              (to the lower / upper neighbour)
 *   cg_begin(d_v, v_lo, v_hi, partial)      b = B V / dt with the
 *                              neighbours' planes of V; r = b, z = D^-1 b
 *   for iter = 0, 1, ... while not done:
 *     cg_direction(iter, all, n_parts, send_lo, send_hi)   convergence test
 *                              on the gathered partials, p = z + beta p, its
 *                              boundary planes into send_lo / send_hi
 *     cg_product(iter, p_lo, p_hi, partial)  q = A p with the neighbours'
 *                              planes of p
 *     cg_update(iter, all, n_parts, partial)  x += alpha p, r -= alpha q,
 *                              z = D^-1 r
 *   cg_end(d_v, t_new)         V = x (activation times at t_new when cells
 *                              are bound)
 * Every part sums the gathered partials in part order, so all parts stop
 * together and the result does not depend on which rank holds which part.
 * Once done, the remaining launches of a chunk return at once: the caller
 * may run several iterations between cg_status calls (blocking; iters is
 * negative when max_iter was reached). */
int cep_part_pack(cep_part_t p, const void *d_v, void *d_lo, void *d_hi);
int cep_part_cg_begin(cep_part_t p, const void *d_v, const void *d_v_lo, const void *d_v_hi, void *d_partial);
int cep_part_cg_direction(cep_part_t p, int iter, const void *d_all, int n_parts, void *d_send_lo, void *d_send_hi);
int cep_part_cg_product(cep_part_t p, int iter, const void *d_p_lo, const void *d_p_hi, void *d_partial);
int cep_part_cg_update(cep_part_t p, int iter, const void *d_all, int n_parts, void *d_partial);
int cep_part_cg_status(cep_part_t p, int iter, int *done, int *iters, double *res);
int cep_part_cg_end(cep_part_t p, void *d_v, double t_new);
/* The part's cells (one instance per owned row, on the part's stream): the
 * tissue's S1 stimulus over the owned rows (mask of n_own bytes, NULL = none)
 * as cep_tissue_set_stimulus, and activation times (first step with
 * V >= act_thr). ionic_step: every owned node's ionic update at tissue time
 * t (Cheart::cellular_reaction, heart.cpp:274-430). */
int cep_part_bind_cells(cep_part_t p, cep_batch_t cells, const unsigned char *s1_mask, double bcl, double t_crt,
                        double dur, int n_pace, double act_thr);
int cep_part_ionic_step(cep_part_t p, double t);
int cep_part_get_activation(cep_part_t p, double *t_act);

#ifdef __cplusplus
}
#endif
#endif
