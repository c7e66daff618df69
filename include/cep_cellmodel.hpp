/*
 * C++ adapters over the cep_b200 C ABI for reference-style callers.
 *
 *  - cep::Cellmodel keeps the shape of the reference's cell-model classes
 *    (DrugSimulation/cellmodels/cellmodel.hpp:4-36 and
 *    CEPCell_NEO/cellmodels/patch_clamp.hpp:4-26): public ALGEBRAIC /
 *    CONSTANTS / RATES / STATES arrays, isS1 / isEctopic, the initConsts
 *    overloads, computeRates(TIME, C, R, S, A) and solveAnalytical(dt). A
 *    driver written against those members (an explicit loop or
 *    Cheart::cellular_reaction, heart.cpp:274-430) runs unchanged on one
 *    device instance. It is a compatibility shim: a population belongs in
 *    one cep::Population (or cep_batch_t), not in n adapters.
 *  - cep::Population is an owning RAII wrapper of one cep_batch_t.
 *
 * Header-only; link with libcep_b200.so. Errors throw cep::Error.
 */
#ifndef CEP_CELLMODEL_HPP
#define CEP_CELLMODEL_HPP

#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "cep_b200.h"

namespace cep {

class Error : public std::runtime_error {
 public:
  Error(int code, const std::string &msg) : std::runtime_error(msg), code(code) {}
  int code;
};

inline void check(int rc) {
  if (rc != CEP_OK) throw Error(rc, cep_last_error());
}

class Population {
 public:
  Population(int model, int n, int precision = CEP_PREC_FP64, void *stream = nullptr) {
    check(cep_batch_create(model, n, precision, stream, &h_));
    check(cep_batch_size(h_, &n_, &ns_));
  }
  ~Population() { cep_batch_destroy(h_); }
  Population(const Population &) = delete;
  Population &operator=(const Population &) = delete;

  cep_batch_t handle() const { return h_; }
  int size() const { return n_; }
  int states_size() const { return ns_; }

  void initConsts(const double *celltype, const double *conc, const double *hill, int hill_stride,
                  unsigned flags = CEP_FLAG_QUIRKS) {
    check(cep_batch_init(h_, celltype, conc, hill, hill_stride, flags));
  }
  void setPacing(double bcl, double stim_start = -1, double stim_dur = -1, double amp_scale = 1) {
    check(cep_batch_set_pacing(h_, bcl, stim_start, stim_dur, amp_scale));
  }
  void setProtocol(double dt, int n_pace, int first_pace, double dt_write = 1.0, double qnet_thr = -1e300) {
    check(cep_batch_set_protocol(h_, dt, n_pace, first_pace, dt_write, qnet_thr));
  }
  /* CONSTANTS[g] *= factor[i] for every instance (CEP_SCALE_*). */
  void scale(int conductance, const double *factor) { check(cep_batch_scale(h_, conductance, factor)); }
  void run(long n_steps) { check(cep_batch_run(h_, n_steps)); }
  void runToEnd(long steps_per_launch = 20000) { check(cep_batch_run_to_end(h_, steps_per_launch)); }
  void step(double t, double dt, int stim_mode = -1) { check(cep_batch_step(h_, t, dt, stim_mode)); }
  std::vector<double> states(int layout = CEP_LAYOUT_AOS) const {
    std::vector<double> s((size_t)n_ * ns_);
    check(cep_batch_get_states(h_, s.data(), layout));
    return s;
  }
  void setStates(const double *s, int layout = CEP_LAYOUT_AOS) { check(cep_batch_set_states(h_, s, layout)); }
  std::vector<cep_biomarkers_t> biomarkers() const {
    std::vector<cep_biomarkers_t> b(n_);
    check(cep_batch_get_biomarkers(h_, b.data()));
    return b;
  }
  /* Fastest kernel form and block size for this population (state kept). */
  void autotune(long n_steps = 400) { check(cep_batch_autotune(h_, n_steps, nullptr, nullptr)); }
  /* The whole population mid-protocol, and its resume (heart.cpp iopt = 1
   * style, but exact). */
  std::vector<unsigned char> checkpoint() const {
    size_t bytes = 0;
    check(cep_batch_checkpoint_size(h_, &bytes));
    std::vector<unsigned char> buf(bytes);
    check(cep_batch_checkpoint(h_, buf.data(), buf.size()));
    return buf;
  }
  void restore(const std::vector<unsigned char> &buf) { check(cep_batch_restore(h_, buf.data(), buf.size())); }
  /* apdr_bench.cpp's dynamic restitution: records [n][max_records]. */
  std::vector<cep_apdr_record_t> restitution(const std::vector<double> &bcl, int n_pace, double dt, int max_records,
                                             int *n_records = nullptr, long steps_per_launch = 20000) {
    std::vector<cep_apdr_record_t> out((size_t)n_ * (size_t)max_records);
    check(cep_batch_restitution(h_, bcl.data(), (int)bcl.size(), n_pace, dt, steps_per_launch, out.data(),
                                max_records, n_records));
    return out;
  }
  /* CEPPatch/benchpatch.cpp's voltage-clamp replay: out [v.size()][n]. */
  std::vector<double> clamp(const std::vector<double> &v, double t0, double dt, int current) {
    std::vector<double> out(v.size() * (size_t)n_);
    check(cep_batch_clamp(h_, v.data(), (long)v.size(), t0, dt, current, out.data()));
    return out;
  }

 private:
  cep_batch_t h_ = nullptr;
  int n_ = 0, ns_ = 0;
};

/* One cell with the reference's member layout (cellmodel.hpp:4-36: the
 * unsigned short sizes, inline 255-entry arrays and the gate / current /
 * concentration index tables), stepped on the device.
 *
 *  - STATES mirrors the device state after every solveAnalytical; edits a
 *    caller makes to STATES (e.g. V from the diffusion solve) are uploaded
 *    before the next computeRates.
 *  - computeRates fills the whole RATES vector (dy/dt of every state, as the
 *    reference's CVODE right-hand side uses it: CEPCell_NEO/modules/
 *    commons.cpp:26-35) for ORd 2011, CiPA-ORd and ToR-ORd, and RATES[0]
 *    for the ten Tusscher models. For ORd 2011 and CiPA-ORd the seven
 *    channel currents are written at the reference's ALGEBRAIC indices
 *    (ORd: INa 62, INaL 64, Ito 70, ICaL 81, IKr 96, IKs 98, IK1 100,
 *    enum_Ohara_Rudy_2011.hpp; CiPA: 58, 60, 66, 83, 90, 96, 98,
 *    enum_ohara_rudy_cipa_v1_2017.hpp), so qNet code reading
 *    ALGEBRAIC[INaL] etc. keeps working; other ALGEBRAIC entries are not
 *    produced.
 *  - For ORd 2011 and CiPA-ORd, CONSTANTS holds the pacing (ORd: BCL 140,
 *    stim_start 139, duration 13, amp 12; CiPA: 15, 12, 16, 14) and the
 *    per-instance conductances (ORd: GNa 42, GNaL 96, Gto 97, PCa 99, GKr
 *    101, GKs 102, GK1 103, GKb 105, Gncx 128, Pnak 138; CiPA: 45, 153,
 *    154, 156, 159, 160, 161, 163, 194, 204) after initConsts. A caller's
 *    write to any of them (cipa_drug_bench.cpp:146-148, heart.cpp:219-222:
 *    CONSTANTS[BCL] = ..., CONSTANTS[amp] *= ..., CONSTANTS[GNa] *= ...)
 *    reaches the device before the next step. Other CONSTANTS entries are
 *    not read. Other models take setPacing() and Population::scale.
 *  - tissue = true reproduces the reference's TISSUE builds: the stimulus is
 *    isS1 (-DTISSUE), else the model's periodic single-cell stimulus. */
class Cellmodel {
 public:
  static constexpr int kArr = 255;
  bool isEctopic = false;
  bool isS1 = false;
  unsigned short algebraic_size = 0, constants_size = 0, states_size = 0;
  unsigned short gates_size = 0, current_size = 0, concs_size = 0;
  double ALGEBRAIC[kArr];
  double CONSTANTS[kArr];
  double RATES[kArr];
  double STATES[kArr];
  char gates_header[kArr];
  unsigned short gates_indices[kArr];
  char current_header[kArr];
  unsigned short current_indices[kArr];
  char concs_header[kArr];
  unsigned short concs_indices[kArr];

  explicit Cellmodel(int model, int precision = CEP_PREC_FP64, bool tissue = false)
      : pop_(model, 1, precision), model_(model), tissue_(tissue) {
    std::memset(ALGEBRAIC, 0, sizeof(ALGEBRAIC));
    std::memset(CONSTANTS, 0, sizeof(CONSTANTS));
    std::memset(RATES, 0, sizeof(RATES));
    std::memset(STATES, 0, sizeof(STATES));
    std::memset(gates_header, 0, sizeof(gates_header));
    std::memset(current_header, 0, sizeof(current_header));
    std::memset(concs_header, 0, sizeof(concs_header));
    std::memset(gates_indices, 0, sizeof(gates_indices));
    std::memset(current_indices, 0, sizeof(current_indices));
    std::memset(concs_indices, 0, sizeof(concs_indices));
    states_size = (unsigned short)pop_.states_size();
    if (model == CEP_MODEL_ORD2011) {  // the DrugSimulation ORd's tables (Ohara_Rudy_2011.cpp:438-453)
      algebraic_size = 198;
      constants_size = 144;
      static const unsigned short g[] = {14, 13, 40, 17, 37, 6,  3,  36, 34, 30, 16, 5,  32, 4,  21,
                                         38, 1,  35, 7,  23, 19, 10, 28, 27, 24, 11, 31, 20, 8,  22};
      static const unsigned short c[] = {16, 67, 30, 187, 157, 168, 169, 73, 178, 150, 135,
                                         42, 1,  9,  26,  49,  147, 143, 17, 184, 36};
      static const unsigned short k[] = {18, 5, 2, 0, 25, 26, 29, 9};
      gates_size = 30;
      current_size = 21;
      concs_size = 8;
      std::memcpy(gates_indices, g, sizeof(g));
      std::memcpy(current_indices, c, sizeof(c));
      std::memcpy(concs_indices, k, sizeof(k));
      std::strncpy(gates_header,
                   "m,j,jp,hf,hs,hsp,mL,hL,hLp,a,ap,ki,iF,iS,iFp,iSp,xrf,xrs,xs1,xs2,xk1,d,ff,fs,fcaf,nca,jca,fca"
                   "     s,ffp,fcafp,",
                   kArr - 1);
      std::strncpy(current_header,
                   "INa,INaL,Ito,IKr,IKs,IK1,ICaL,ICaNa,ICaK,INaCa_ss,INaK,Jdiff,JdiffK,JdiffNa,Jup,Jrel,Jtr,"
                   "     ,IpCa,ICab,INab,IKb",
                   kArr - 1);
      std::strncpy(concs_header, "nai,ki,cass,nass,cai,kss,CaMKT,cansr,cajsr", kArr - 1);
    }
  }
  virtual ~Cellmodel() {}

  virtual void initConsts() { init(0.0, 0.0, nullptr, false); }
  virtual void initConsts(double type) { init(type, 0.0, nullptr, false); }
  virtual void initConsts(double type, bool is_dutta) { init(type, 0.0, nullptr, is_dutta); }
  virtual void initConsts(double type, double conc, double *hill) { init(type, conc, hill, false); }
  virtual void initConsts(double type, double conc, double *hill, bool is_dutta) { init(type, conc, hill, is_dutta); }
  /* The bootstrap overload of the reference's base class, which no model
   * of the reference overrides: it does nothing there and here. */
  virtual void initConsts(double type, double conc, double *hill, double *boot) {
    (void)type; (void)conc; (void)hill; (void)boot;
  }

  virtual void computeRates(double TIME, double *C, double *R, double *S, double *A) {
    if (C != CONSTANTS) std::memcpy(CONSTANTS, C, sizeof(CONSTANTS));
    sync_in(S);
    sync_consts();
    double dvdt = 0, cur[7] = {0};
    check(cep_batch_rates(pop_.handle(), TIME, &dvdt, cur));
    if (model_ == CEP_MODEL_ORD2011 || model_ == CEP_MODEL_CIPA2017 || model_ == CEP_MODEL_TOMEK2019) {
      check(cep_batch_rates_all(pop_.handle(), TIME, R));
    } else {
      R[0] = dvdt;
    }
    const int *idx = alg_index();
    if (idx)
      for (int k = 0; k < 7; ++k) A[idx[k]] = cur[k];
    t_ = TIME;
  }

  virtual void solveAnalytical(double dt) {
    sync_in(STATES);
    sync_consts();
    pop_.step(t_, dt, tissue_ ? (isS1 ? 1 : 0) : -1);
    sync_out();
  }
  /* The reference's base class declares an RK4 step that no model
   * implements (DrugSimulation/modules/drug_sim.cpp:227 calls it); like
   * there, it does nothing. */
  virtual void solveRK4(double TIME, double dt) { (void)TIME; (void)dt; }

  /* Pacing for every model (BCL, stimulus start and duration in ms; the
   * amplitude as a factor on the model default). */
  void setPacing(double bcl, double stim_start = -1, double stim_dur = -1, double amp_scale = 1) {
    pop_.setPacing(bcl, stim_start, stim_dur, amp_scale);
    const int *p = pacing_index();
    if (p) {
      CONSTANTS[p[0]] = bcl;
      if (stim_start >= 0) CONSTANTS[p[1]] = stim_start;
      if (stim_dur >= 0) CONSTANTS[p[2]] = stim_dur;
      CONSTANTS[p[3]] *= amp_scale;
      remember();
    }
  }

  Population &population() { return pop_; }

 private:
  // CONSTANTS indices of BCL, stim_start, duration, amp
  const int *pacing_index() const {
    static const int ord[4] = {140, 139, 13, 12}, cipa[4] = {15, 12, 16, 14};
    return model_ == CEP_MODEL_ORD2011 ? ord : model_ == CEP_MODEL_CIPA2017 ? cipa : nullptr;
  }
  // ALGEBRAIC indices of INa, INaL, Ito, ICaL, IKr, IKs, IK1
  const int *alg_index() const {
    static const int ord[7] = {62, 64, 70, 81, 96, 98, 100}, cipa[7] = {58, 60, 66, 83, 90, 96, 98};
    return model_ == CEP_MODEL_ORD2011 ? ord : model_ == CEP_MODEL_CIPA2017 ? cipa : nullptr;
  }
  // CONSTANTS indices of the CEP_SCALE_* conductances (-1: not mirrored)
  const int *conductance_index() const {
    static const int ord[CEP_SCALE_COUNT] = {42, 96, 97, 99, 101, 102, 103, -1, -1, -1, -1, 105, 128, 138};
    static const int cipa[CEP_SCALE_COUNT] = {45, 153, 154, 156, 159, 160, 161, -1, -1, -1, -1, 163, 194, 204};
    return model_ == CEP_MODEL_ORD2011 ? ord : model_ == CEP_MODEL_CIPA2017 ? cipa : nullptr;
  }
  void init(double type, double conc, double *hill, bool is_dutta) {
    double ct = type, cc = conc;
    pop_.initConsts(&ct, &cc, hill, hill ? (model_ == CEP_MODEL_CIPA2017 ? CEP_HILL_WIDTH : 14) : 0,
                    CEP_FLAG_QUIRKS | (is_dutta ? CEP_FLAG_DUTTA : 0u));
    if (const int *p = pacing_index()) {  // initConsts defaults (Ohara_Rudy_2011.cpp:494-678)
      CONSTANTS[p[0]] = 1000.0;
      CONSTANTS[p[1]] = 10.0;
      CONSTANTS[p[2]] = 0.5;
      CONSTANTS[p[3]] = -80.0;
    }
    if (const int *g = conductance_index())
      for (int k = 0; k < CEP_SCALE_COUNT; ++k)
        if (g[k] >= 0) check(cep_batch_get_conductance(pop_.handle(), k, &CONSTANTS[g[k]]));
    remember();
    sync_out();
  }
  void remember() { std::memcpy(consts_seen_, CONSTANTS, sizeof(CONSTANTS)); }
  // uploads what a caller changed in the mirrored CONSTANTS entries
  void sync_consts() {
    const int *p = pacing_index();
    if (!p) return;
    bool pacing = false;
    for (int k = 0; k < 4; ++k) pacing |= CONSTANTS[p[k]] != consts_seen_[p[k]];
    if (pacing) {
      const double scale = consts_seen_[p[3]] != 0.0 ? CONSTANTS[p[3]] / consts_seen_[p[3]] : 1.0;
      check(cep_batch_set_pacing(pop_.handle(), CONSTANTS[p[0]], CONSTANTS[p[1]], CONSTANTS[p[2]], scale));
    }
    const int *g = conductance_index();
    for (int k = 0; k < CEP_SCALE_COUNT; ++k)
      if (g[k] >= 0 && CONSTANTS[g[k]] != consts_seen_[g[k]])
        check(cep_batch_set_conductance(pop_.handle(), k, &CONSTANTS[g[k]]));
    remember();
  }
  void sync_in(const double *S) {
    if (S != STATES) std::memcpy(STATES, S, sizeof(double) * states_size);
    if (std::memcmp(STATES, shadow_, sizeof(double) * states_size) != 0) {
      pop_.setStates(STATES);
      std::memcpy(shadow_, STATES, sizeof(double) * states_size);
    }
  }
  void sync_out() {
    check(cep_batch_get_states(pop_.handle(), STATES, CEP_LAYOUT_AOS));
    std::memcpy(shadow_, STATES, sizeof(double) * states_size);
  }

  Population pop_;
  int model_;
  bool tissue_;
  double t_ = 0.0;
  double consts_seen_[kArr] = {0};
  double shadow_[kArr] = {0};
};

}  // namespace cep

#endif
