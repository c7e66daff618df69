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

/* One cell with the reference's member layout, stepped on the device.
 *
 *  - STATES mirrors the device state after every solveAnalytical; edits a
 *    caller makes to STATES (e.g. V from the diffusion solve) are uploaded
 *    before the next computeRates.
 *  - computeRates fills RATES[0] (dV/dt) and, for ORd 2011, the seven
 *    channel currents at the reference's ALGEBRAIC indices (INa 62, INaL 64,
 *    Ito 70, ICaL 81, IKr 96, IKs 98, IK1 100: enum_Ohara_Rudy_2011.hpp), so
 *    qNet code reading ALGEBRAIC[INaL] etc. keeps working; the other RATES
 *    and ALGEBRAIC entries are not produced.
 *  - For ORd 2011, CONSTANTS[BCL] (140), [stim_start] (139), [duration] (13)
 *    and [amp] (12) hold the pacing and a caller's writes to them reach the
 *    device before the next step (cipa_drug_bench.cpp:146-147 style); other
 *    models take setPacing().
 *  - tissue = true reproduces the reference's TISSUE builds: the stimulus is
 *    isS1 (-DTISSUE), else the model's periodic single-cell stimulus. */
class Cellmodel {
 public:
  static constexpr int kArr = 255;
  double ALGEBRAIC[kArr];
  double CONSTANTS[kArr];
  double RATES[kArr];
  double STATES[kArr];
  bool isS1 = false;
  bool isEctopic = false;
  unsigned int algebraic_size = 0, constants_size = 0, states_size = 0;

  explicit Cellmodel(int model, int precision = CEP_PREC_FP64, bool tissue = false)
      : pop_(model, 1, precision), model_(model), tissue_(tissue) {
    std::memset(ALGEBRAIC, 0, sizeof(ALGEBRAIC));
    std::memset(CONSTANTS, 0, sizeof(CONSTANTS));
    std::memset(RATES, 0, sizeof(RATES));
    std::memset(STATES, 0, sizeof(STATES));
    states_size = (unsigned)pop_.states_size();
  }
  virtual ~Cellmodel() {}

  virtual void initConsts() { init(0.0, 0.0, nullptr, false); }
  virtual void initConsts(double type) { init(type, 0.0, nullptr, false); }
  virtual void initConsts(double type, bool is_dutta) { init(type, 0.0, nullptr, is_dutta); }
  virtual void initConsts(double type, double conc, double *hill) { init(type, conc, hill, false); }
  virtual void initConsts(double type, double conc, double *hill, bool is_dutta) { init(type, conc, hill, is_dutta); }

  virtual void computeRates(double TIME, double *C, double *R, double *S, double *A) {
    (void)C;
    sync_in(S);
    sync_pacing();
    double dvdt = 0, cur[7] = {0};
    check(cep_batch_rates(pop_.handle(), TIME, &dvdt, cur));
    R[0] = dvdt;
    if (model_ == CEP_MODEL_ORD2011) {
      static const int idx[7] = {62, 64, 70, 81, 96, 98, 100};  // INa INaL Ito ICaL IKr IKs IK1
      for (int k = 0; k < 7; ++k) A[idx[k]] = cur[k];
    }
    t_ = TIME;
  }

  virtual void solveAnalytical(double dt) {
    sync_in(STATES);
    sync_pacing();
    pop_.step(t_, dt, tissue_ ? (isS1 ? 1 : 0) : -1);
    sync_out();
  }

  /* Pacing for every model (BCL, stimulus start and duration in ms; the
   * amplitude as a factor on the model default). */
  void setPacing(double bcl, double stim_start = -1, double stim_dur = -1, double amp_scale = 1) {
    pop_.setPacing(bcl, stim_start, stim_dur, amp_scale);
    if (model_ == CEP_MODEL_ORD2011) {
      CONSTANTS[140] = bcl;
      if (stim_start >= 0) CONSTANTS[139] = stim_start;
      if (stim_dur >= 0) CONSTANTS[13] = stim_dur;
      CONSTANTS[12] *= amp_scale;
      remember_pacing();
    }
  }

  Population &population() { return pop_; }

 private:
  void init(double type, double conc, double *hill, bool is_dutta) {
    double ct = type, cc = conc;
    pop_.initConsts(&ct, &cc, hill, hill ? (model_ == CEP_MODEL_CIPA2017 ? CEP_HILL_WIDTH : 14) : 0,
                    CEP_FLAG_QUIRKS | (is_dutta ? CEP_FLAG_DUTTA : 0u));
    if (model_ == CEP_MODEL_ORD2011) {  // Ohara_Rudy_2011.cpp initConsts defaults
      CONSTANTS[140] = 1000.0;
      CONSTANTS[139] = 10.0;
      CONSTANTS[13] = 0.5;
      CONSTANTS[12] = -80.0;
      remember_pacing();
    }
    sync_out();
  }
  void remember_pacing() {
    pacing_[0] = CONSTANTS[140];
    pacing_[1] = CONSTANTS[139];
    pacing_[2] = CONSTANTS[13];
    pacing_[3] = CONSTANTS[12];
  }
  void sync_pacing() {
    if (model_ != CEP_MODEL_ORD2011) return;
    if (CONSTANTS[140] == pacing_[0] && CONSTANTS[139] == pacing_[1] && CONSTANTS[13] == pacing_[2] &&
        CONSTANTS[12] == pacing_[3])
      return;
    const double scale = pacing_[3] != 0.0 ? CONSTANTS[12] / pacing_[3] : 1.0;
    check(cep_batch_set_pacing(pop_.handle(), CONSTANTS[140], CONSTANTS[139], CONSTANTS[13], scale));
    remember_pacing();
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
  double pacing_[4] = {0, 0, 0, 0};
  double shadow_[kArr] = {0};
};

}  // namespace cep

#endif
