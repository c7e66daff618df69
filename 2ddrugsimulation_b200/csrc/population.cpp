// One screening job end to end: the CiPA bench's sample x concentration loop
// (CEPCell_NEO/modules/cipa_drug_bench.cpp:128-380) for a whole population,
// as batches on the device, with the mixed path's accuracy bar kept for
// every instance.
//
// Mixed precision holds APD90 / CaD90 to 0.1 ms and qNet to 1 % of the FP64
// path for instances that repolarise. Instances that a drug depolarises
// (diastolic Vm above about -80 mV) cross their 90 % level at ~0.1 mV/ms:
// their APD90 moves by tenths of a ms under relative perturbations of 1e-5,
// which FP32 gates cannot hold. Such instances run in FP64 instead:
//   1. every instance runs `screen_paces` paces in mixed precision;
//   2. those whose membrane potential at the end of the screening (the
//      diastolic Vm before the next stimulus) is above refine_above_vm
//      start again from their initial state in an FP64 batch on a second
//      stream, concurrently with the mixed batch's remaining paces;
//   3. an instance whose evaluated record still shows a diastolic Vm above
//      the threshold, an APD90 above 0.9 BCL or an intermittent rhythm
//      (some evaluated beats with an action potential at the peak sample
//      and some without: a cell at the edge of 2:1 block, whose
//      beat-to-beat dynamics can settle into different regimes under FP32
//      and FP64 rounding) runs again in FP64 after both batches finish. A
//      cell whose upstroke misses the peak sample in every beat (a strong
//      sodium block) has no APD in either precision and is not re-run.
// The FP64 records replace the mixed ones; refined[i] says which path
// produced instance i's record.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "../../include/cep_b200.h"
#include "internal.h"

namespace {

struct Stream {
  cudaStream_t s = nullptr;
  ~Stream() {
    if (s) cudaStreamDestroy(s);
  }
};

struct Batch {
  cep_batch_t b = nullptr;
  ~Batch() {
    if (b) cep_batch_destroy(b);
  }
};

int fail(int code, const char *msg) { return cep_internal_set_fail(code, msg); }

// A batch of the instances idx (all when idx is empty) at the start of the
// job's protocol.
int make_batch(const cep_population_job_t *j, int precision, const std::vector<int> &idx, cudaStream_t st,
               Batch &out) {
  const int n = idx.empty() ? j->n : (int)idx.size();
  std::vector<double> ct, cc, hh;
  const double *pct = j->celltype, *pcc = j->conc, *phh = j->hill;
  if (!idx.empty()) {
    ct.resize(n);
    cc.resize(n);
    if (j->hill) hh.resize((size_t)n * j->hill_stride);
    for (int k = 0; k < n; ++k) {
      ct[k] = j->celltype ? j->celltype[idx[k]] : 0.0;
      cc[k] = j->conc ? j->conc[idx[k]] : 0.0;
      if (j->hill) std::memcpy(&hh[(size_t)k * j->hill_stride], j->hill + (size_t)idx[k] * j->hill_stride,
                               sizeof(double) * j->hill_stride);
    }
    pct = ct.data();
    pcc = cc.data();
    phh = j->hill ? hh.data() : nullptr;
  }
  int rc;
  if ((rc = cep_batch_create(j->model, n, precision, st, &out.b))) return rc;
  if ((rc = cep_batch_init(out.b, pct, pcc, phh, j->hill_stride, j->flags))) return rc;
  if ((rc = cep_batch_set_pacing(out.b, j->bcl, -1.0, -1.0, j->amp_scale))) return rc;
  if (j->scale)
    for (int g = 0; g < CEP_SCALE_COUNT; ++g) {
      std::vector<double> f(n);
      bool any = false;
      for (int k = 0; k < n; ++k) {
        f[k] = j->scale[(size_t)(idx.empty() ? k : idx[k]) * CEP_SCALE_COUNT + g];
        any |= f[k] != 1.0;
      }
      if (any && (rc = cep_batch_scale(out.b, g, f.data()))) return rc;
    }
  if (j->states_init) {
    int ns = 0;
    cep_batch_size(out.b, nullptr, &ns);
    std::vector<double> y((size_t)n * ns);
    for (int k = 0; k < n; ++k) std::memcpy(&y[(size_t)k * ns], j->states_init, sizeof(double) * ns);
    if ((rc = cep_batch_set_states(out.b, y.data(), CEP_LAYOUT_AOS))) return rc;
  }
  return cep_batch_set_protocol(out.b, j->dt, j->n_pace, j->first_pace, j->dt_write, -1e300);
}

// Launches that take a batch from step `done` to the end of its protocol
// (imax = (int)((n_pace * BCL) / dt) steps, cipa_drug_bench.cpp:188, plus
// the launch that marks the instances done).
long launches_left(const cep_population_job_t *j, long done, long spl) {
  const long imax = (long)((j->n_pace * j->bcl) / j->dt);
  return (imax - done + spl) / spl + 1;
}

}  // namespace

extern "C" int cep_population_late_mask(const cep_biomarkers_t *recs, int n, double refine_above_vm, double bcl,
                                        int evaluated, int *mask) {
  if (n < 0 || (n > 0 && (!recs || !mask))) return fail(CEP_ERR_ARG, "null records or mask");
  if (!(bcl > 0) || evaluated < 0) return fail(CEP_ERR_ARG, "bcl must be positive and evaluated >= 0");
  constexpr double kNearBlock = 0.9;  // APD90 / BCL above which a beat is at the edge of block
  for (int i = 0; i < n; ++i) {
    const cep_biomarkers_t &r = recs[i];
    mask[i] = (!(r.vm_valley < refine_above_vm) || r.apd90 > kNearBlock * bcl ||
               (r.n_eligible > 0 && r.n_eligible < evaluated))
                  ? 1
                  : 0;
  }
  return CEP_OK;
}

extern "C" int cep_population_run(const cep_population_job_t *j, cep_biomarkers_t *out, int *refined) {
  if (!j || !out) return fail(CEP_ERR_ARG, "null argument");
  if (j->n <= 0 || !(j->bcl > 0) || !(j->dt > 0) || j->n_pace <= 0)
    return fail(CEP_ERR_ARG, "n, bcl, dt and n_pace must be positive");
  if (j->precision != CEP_PREC_FP64 && j->precision != CEP_PREC_MIXED) return fail(CEP_ERR_ARG, "bad precision");
  const long spl = j->steps_per_launch > 0 ? j->steps_per_launch : 20000;
  const bool refine = j->precision == CEP_PREC_MIXED && std::isfinite(j->refine_above_vm);
  if (cep_device_count() == 0) return fail(CEP_ERR_NO_DEVICE, "no CUDA device visible");
  std::vector<int> how(j->n, 0);
  Stream sa, sb;
  if (cudaStreamCreateWithFlags(&sa.s, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&sb.s, cudaStreamNonBlocking) != cudaSuccess)
    return fail(CEP_ERR_CUDA, "stream creation failed");
  Batch a;
  int rc = make_batch(j, j->precision, {}, sa.s, a);
  if (rc) return rc;
  long done = 0;
  std::vector<int> cand;
  Batch b;
  int ns = 0;
  cep_batch_size(a.b, nullptr, &ns);
  if (refine) {  // 1. screening paces in mixed precision
    const long steps_per_bcl = (long)(j->bcl / j->dt);
    const long screen = (long)std::max(1, j->screen_paces) * steps_per_bcl;
    for (long s = 0; s < screen; s += spl)
      if ((rc = cep_batch_run(a.b, std::min(spl, screen - s)))) return rc;
    done = screen;
    std::vector<double> y((size_t)ns * j->n);
    if ((rc = cep_batch_get_states(a.b, y.data(), CEP_LAYOUT_SOA))) return rc;
    for (int i = 0; i < j->n; ++i)
      if (!(y[i] < j->refine_above_vm)) cand.push_back(i);  // row 0 of the SoA block is V
    // 2. the candidates in FP64 from their initial state, on the second stream
    if (!cand.empty() && (rc = make_batch(j, CEP_PREC_FP64, cand, sb.s, b))) return rc;
  }
  // the two batches' launches interleaved: both streams stay busy
  long la = launches_left(j, done, spl), lb = b.b ? launches_left(j, 0, spl) : 0;
  while (la > 0 || lb > 0) {
    if (la-- > 0 && (rc = cep_batch_run(a.b, spl))) return rc;
    if (lb-- > 0 && (rc = cep_batch_run(b.b, spl))) return rc;
  }
  if ((rc = cep_batch_run_to_end(a.b, spl))) return rc;  // no-op once every instance is done
  if ((rc = cep_batch_get_biomarkers(a.b, out))) return rc;
  if (b.b) {
    if ((rc = cep_batch_run_to_end(b.b, spl))) return rc;
    std::vector<cep_biomarkers_t> r(cand.size());
    if ((rc = cep_batch_get_biomarkers(b.b, r.data()))) return rc;
    for (size_t k = 0; k < cand.size(); ++k) {
      out[cand[k]] = r[k];
      how[cand[k]] = 1;
    }
  }
  if (refine) {  // 3. whatever the screening missed
    std::vector<int> late, mask(j->n);
    const int evaluated = j->first_pace >= 0 ? std::max(0, j->n_pace - j->first_pace) : 0;
    if ((rc = cep_population_late_mask(out, j->n, j->refine_above_vm, j->bcl, evaluated, mask.data()))) return rc;
    for (int i = 0; i < j->n; ++i)
      if (how[i] == 0 && mask[i]) late.push_back(i);
    if (!late.empty()) {
      Batch c;
      if ((rc = make_batch(j, CEP_PREC_FP64, late, sb.s, c))) return rc;
      if ((rc = cep_batch_run_to_end(c.b, spl))) return rc;
      std::vector<cep_biomarkers_t> r(late.size());
      if ((rc = cep_batch_get_biomarkers(c.b, r.data()))) return rc;
      for (size_t k = 0; k < late.size(); ++k) {
        out[late[k]] = r[k];
        how[late[k]] = 2;
      }
    }
  }
  if (refined) std::memcpy(refined, how.data(), sizeof(int) * j->n);
  return CEP_OK;
}
