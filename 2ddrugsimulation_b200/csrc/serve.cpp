// Screening-job server with continuous batching: the cep_serve_* C ABI
// (include/cep_b200.h). No counterpart in the reference, which runs one job
// per MPI process (cipa_drug_bench.cpp).
//
// One resident batch is a pool of slots in HBM. A job is a list of
// instances (samples x concentrations, each with its Hill row) and occupies
// a contiguous slot range from admission to completion. A scheduler thread
// loops:
//   1. admit queued jobs, in arrival order, into the first free range that
//      fits (a later, smaller job may pass a larger one that does not fit
//      yet); admission initialises, paces and starts only that range;
//   2. launch one run of K steps over the whole pool: every running slot
//      advances, whatever job it belongs to and wherever that job is in its
//      protocol; idle and finished slots return at once;
//   3. read the per-slot status words; a job whose slots are all finished
//      has its biomarkers collected and its range released.
// Each instance's arithmetic does not depend on its neighbours, so a job's
// results are bit-identical alone or in any mix.
//
// Tissue-patch jobs (2D TT2006 sheets) get their own cells, operator and
// tissue on a second stream, admitted against the HBM budget left after the
// pool; each round the running patches advance together as one tissue group
// (one batched PCG launch per step) while the pool's launch runs, so the two
// kinds of work overlap on the device.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/cep_b200.h"
#include "internal.h"

namespace {

using Clock = std::chrono::steady_clock;

struct Job {
  uint64_t id = 0;
  bool tissue = false;
  int n = 0;
  std::vector<double> celltype, conc, hill;
  int hill_stride = 0;
  double bcl = 1000.0;
  int n_pace = 1, first_pace = 0;
  unsigned flags = 0;
  int first = -1;  // slot range while admitted
  int state = CEP_JOB_QUEUED;
  bool cancel = false;  // set by cep_serve_cancel; a running job leaves at the next round boundary
  int error = CEP_OK;
  std::string msg;  // the scheduler thread's error message when failed
  std::vector<cep_biomarkers_t> result;
  Clock::time_point t_submit, t_admit, t_done;
  long long steps = 0;  // instance-steps of the whole job
  // tissue patch
  cep_tissue_job_t tj{};
  std::vector<double> thill;
  cep_batch_t cells = nullptr;
  cep_fem_t fem = nullptr;
  cep_tissue_t tis = nullptr;
  long t_total = 0, t_done_steps = 0;
  size_t bytes = 0;
  std::vector<double> v, tact;
};

// device bytes a tissue patch of n nodes may take (cells, operator in all
// formats, work vectors), a generous bound for admission
size_t tissue_bytes(int n) { return (size_t)n * 2048 + ((size_t)4 << 20); }

int fail_fmt(int code, const char *fmt, ...) {
  char buf[256];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  return cep_internal_set_fail(code, buf);
}

double ms_between(Clock::time_point a, Clock::time_point b) {
  return std::chrono::duration<double, std::milli>(b - a).count();
}

}  // namespace

struct cep_server {
  int model = 0, precision = 0, capacity = 0;
  double dt = 0.005, dt_write = 1.0;
  int max_per_beat = 0;
  long steps_per_launch = 10000;
  cep_batch_t pool = nullptr;
  std::vector<int> owner;  // slot occupied (1) or free (-1)
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<std::shared_ptr<Job>> queue;
  std::map<uint64_t, std::shared_ptr<Job>> jobs;
  std::vector<std::shared_ptr<Job>> running;
  uint64_t next_id = 1;
  bool stop = false;
  int fatal = CEP_OK;
  std::thread worker;
  long long launches = 0, steps_done = 0, completed = 0;
  Clock::time_point t_start;
  double busy_ms = 0.0;
  // tissue patches
  cudaStream_t tstream = nullptr;
  std::deque<std::shared_ptr<Job>> tqueue;
  std::vector<std::shared_ptr<Job>> trunning;
  cep_tissue_group_t group = nullptr;
  bool group_dirty = false;
  size_t tissue_budget = 0, tissue_used = 0;
  long tissue_steps_per_round = 200;
  int max_tissues = 64;
};

namespace {

// first free contiguous range of n slots
int find_range(const std::vector<int> &owner, int n) {
  int run = 0;
  for (int i = 0; i < (int)owner.size(); ++i) {
    run = owner[i] < 0 ? run + 1 : 0;
    if (run == n) return i - n + 1;
  }
  return -1;
}

int admit(cep_server *s, Job &j) {
  int rc;
  if ((rc = cep_batch_init_range(s->pool, j.first, j.n, j.celltype.empty() ? nullptr : j.celltype.data(),
                                 j.conc.data(), j.hill.empty() ? nullptr : j.hill.data(), j.hill_stride, j.flags)))
    return rc;
  if ((rc = cep_batch_set_pacing_range(s->pool, j.first, j.n, j.bcl, -1.0, -1.0, 1.0))) return rc;
  return cep_batch_start_range(s->pool, j.first, j.n, j.n_pace, j.first_pace);
}

void tissue_free(Job &j) {
  if (j.tis) cep_tissue_destroy(j.tis);
  if (j.fem) cep_fem_destroy(j.fem);
  if (j.cells) cep_batch_destroy(j.cells);
  j.tis = nullptr;
  j.fem = nullptr;
  j.cells = nullptr;
}

int tissue_admit(cep_server *s, Job &j) {
  const cep_tissue_job_t &q = j.tj;
  const int n = q.nx * q.ny;
  int rc;
  if ((rc = cep_batch_create(CEP_MODEL_TT2006, n, s->precision, s->tstream, &j.cells))) return rc;
  std::vector<double> conc((size_t)n, q.conc), hill;
  if (!j.thill.empty()) {
    hill.resize((size_t)n * 14);
    for (int i = 0; i < n; ++i) std::copy(j.thill.begin(), j.thill.end(), hill.begin() + (size_t)i * 14);
  }
  if ((rc = cep_batch_init(j.cells, nullptr, conc.data(), hill.empty() ? nullptr : hill.data(), 14, CEP_FLAG_QUIRKS)))
    return rc;
  const std::vector<double> D((size_t)(q.nx - 1) * (q.ny - 1), q.D);  // one value per element
  if ((rc = cep_fem_create_grid(2, q.nx, q.ny, 1, q.h, q.dt, D.data(), 1, CEP_FEM_CLASSED, s->tstream, &j.fem)))
    return rc;
  if ((rc = cep_fem_set_solver(j.fem, q.rtol > 0 ? q.rtol : 1e-8, 10000, 1))) return rc;
  if ((rc = cep_tissue_create(j.cells, j.fem, q.dt, &j.tis))) return rc;
  std::vector<unsigned char> mask((size_t)n, 0);
  for (int y = 0; y < std::min(q.stim_ny, q.ny); ++y)
    for (int x = 0; x < std::min(q.stim_nx, q.nx); ++x) mask[(size_t)y * q.nx + x] = 1;
  const int n_pace = (int)std::ceil(q.duration / q.bcl);
  return cep_tissue_set_stimulus(j.tis, mask.data(), q.bcl, 0.0, 1.0, std::max(1, n_pace));
}

void fail_all(cep_server *s, int rc) {
  s->fatal = rc;
  const std::string msg = cep_last_error();
  for (auto *list : {&s->running, &s->trunning})
    for (auto &j : *list) j->msg = msg;
  for (auto *list : {&s->queue, &s->tqueue})
    for (auto &j : *list) j->msg = msg;
  for (auto &j : s->running) {
    j->state = CEP_JOB_FAILED;
    j->error = rc;
  }
  for (auto &j : s->queue) {
    j->state = CEP_JOB_FAILED;
    j->error = rc;
  }
  for (auto *list : {&s->trunning}) {
    for (auto &j : *list) {
      j->state = CEP_JOB_FAILED;
      j->error = rc;
    }
  }
  for (auto &j : s->tqueue) {
    j->state = CEP_JOB_FAILED;
    j->error = rc;
  }
  s->running.clear();
  s->queue.clear();
  s->tqueue.clear();
  s->stop = true;
  s->cv_done.notify_all();
}

void worker_loop(cep_server *s) {
  std::vector<int32_t> status(s->capacity);
  for (;;) {
    std::vector<std::shared_ptr<Job>> admitted, tadmitted;
    {
      std::unique_lock<std::mutex> lock(s->mu);
      s->cv_work.wait(lock, [&] {
        return s->stop || !s->queue.empty() || !s->running.empty() || !s->tqueue.empty() || !s->trunning.empty();
      });
      if (s->stop) return;
      for (auto it = s->queue.begin(); it != s->queue.end();) {
        const int first = find_range(s->owner, (*it)->n);
        if (first < 0) {
          ++it;
          continue;
        }
        (*it)->first = first;
        for (int k = 0; k < (*it)->n; ++k) s->owner[first + k] = 1;
        admitted.push_back(*it);
        it = s->queue.erase(it);
      }
      for (auto it = s->tqueue.begin(); it != s->tqueue.end();) {
        if (s->tissue_used + (*it)->bytes > s->tissue_budget ||
            (int)(s->trunning.size() + tadmitted.size()) >= s->max_tissues) {
          ++it;
          continue;
        }
        s->tissue_used += (*it)->bytes;
        tadmitted.push_back(*it);
        it = s->tqueue.erase(it);
      }
    }
    for (auto &j : admitted) {
      const int rc = admit(s, *j);
      std::lock_guard<std::mutex> lock(s->mu);
      j->t_admit = Clock::now();
      if (rc) {
        j->state = CEP_JOB_FAILED;
        j->error = rc;
        j->msg = cep_last_error();
        for (int k = 0; k < j->n; ++k) s->owner[j->first + k] = -1;
        cep_batch_release_range(s->pool, j->first, j->n);
        s->cv_done.notify_all();
      } else {
        j->state = CEP_JOB_RUNNING;
        s->running.push_back(j);
      }
    }
    for (auto &j : tadmitted) {
      const int rc = tissue_admit(s, *j);
      std::lock_guard<std::mutex> lock(s->mu);
      j->t_admit = Clock::now();
      if (rc) {
        j->msg = cep_last_error();
        tissue_free(*j);
        s->tissue_used -= j->bytes;
        j->state = CEP_JOB_FAILED;
        j->error = rc;
        s->cv_done.notify_all();
      } else {
        j->state = CEP_JOB_RUNNING;
        s->trunning.push_back(j);
        s->group_dirty = true;
      }
    }
    bool have_pop = false;
    std::vector<std::shared_ptr<Job>> tl;
    {
      std::lock_guard<std::mutex> lock(s->mu);
      have_pop = !s->running.empty();
      tl = s->trunning;
    }
    if (!have_pop && tl.empty()) continue;
    const auto t0 = Clock::now();
    int rc = CEP_OK;
    long k_t = 0;
    if (have_pop) rc = cep_batch_run(s->pool, s->steps_per_launch);
    if (!rc && !tl.empty()) {
      if (s->group_dirty) {
        if (s->group) cep_tissue_group_destroy(s->group);
        s->group = nullptr;
        std::vector<cep_tissue_t> ts;
        for (auto &j : tl) ts.push_back(j->tis);
        rc = cep_tissue_group_create(ts.data(), (int)ts.size(), &s->group);
        s->group_dirty = false;
      }
      k_t = s->tissue_steps_per_round;
      for (auto &j : tl) k_t = std::min(k_t, j->t_total - j->t_done_steps);
      if (!rc && k_t > 0) rc = cep_tissue_group_run(s->group, k_t);
    }
    if (!rc && have_pop) rc = cep_batch_get_status(s->pool, status.data());
    if (!rc && !tl.empty() && cudaStreamSynchronize(s->tstream) != cudaSuccess)
      rc = cep_internal_set_fail(CEP_ERR_CUDA, "tissue stream failed");
    const auto t1 = Clock::now();
    std::lock_guard<std::mutex> lock(s->mu);
    s->busy_ms += ms_between(t0, t1);
    s->launches += 1;
    if (rc) {  // the device is unusable: fail every job and stop
      fail_all(s, rc);
      return;
    }
    // cancelled jobs leave between launches: their slots return to the pool,
    // a patch's cells and operator are freed and the tissue group is rebuilt
    for (auto it = s->running.begin(); it != s->running.end();) {
      Job &j = **it;
      if (!j.cancel) {
        ++it;
        continue;
      }
      cep_batch_release_range(s->pool, j.first, j.n);
      for (int k = 0; k < j.n; ++k) s->owner[j.first + k] = -1;
      j.t_done = Clock::now();
      j.state = CEP_JOB_CANCELLED;
      it = s->running.erase(it);
      s->cv_done.notify_all();
    }
    for (auto it = s->trunning.begin(); it != s->trunning.end();) {
      Job &j = **it;
      if (!j.cancel) {
        ++it;
        continue;
      }
      tissue_free(j);
      s->tissue_used -= j.bytes;
      j.t_done = Clock::now();
      j.state = CEP_JOB_CANCELLED;
      s->group_dirty = true;
      it = s->trunning.erase(it);
      s->cv_done.notify_all();
    }
    for (auto it = s->running.begin(); it != s->running.end() && have_pop;) {
      Job &j = **it;
      bool done = true;
      for (int k = 0; k < j.n && done; ++k) done = status[j.first + k] != CEP_INST_RUNNING;
      if (!done) {
        ++it;
        continue;
      }
      j.result.resize(j.n);
      int rc2 = CEP_OK;
      if (j.first_pace >= 0) {
        rc2 = cep_batch_get_biomarkers_range(s->pool, j.first, j.n, j.result.data());
      } else {
        for (int k = 0; k < j.n; ++k) {
          std::memset(&j.result[k], 0, sizeof(cep_biomarkers_t));
          j.result[k].status = status[j.first + k];
        }
      }
      cep_batch_release_range(s->pool, j.first, j.n);
      for (int k = 0; k < j.n; ++k) s->owner[j.first + k] = -1;
      j.t_done = Clock::now();
      j.state = rc2 ? CEP_JOB_FAILED : CEP_JOB_DONE;
      j.error = rc2;
      s->steps_done += j.steps;
      s->completed += 1;
      it = s->running.erase(it);
      s->cv_done.notify_all();
    }
    for (auto it = s->trunning.begin(); it != s->trunning.end();) {
      Job &j = **it;
      j.t_done_steps += k_t;
      if (j.t_done_steps < j.t_total) {
        ++it;
        continue;
      }
      const int n = j.tj.nx * j.tj.ny;
      j.v.resize(n);
      j.tact.resize(n);
      int rc2 = cep_tissue_get_v(j.tis, j.v.data());
      if (!rc2) rc2 = cep_tissue_get_activation(j.tis, j.tact.data());
      if (rc2) j.msg = cep_last_error();
      tissue_free(j);
      s->tissue_used -= j.bytes;
      j.t_done = Clock::now();
      j.state = rc2 ? CEP_JOB_FAILED : CEP_JOB_DONE;
      j.error = rc2;
      s->steps_done += j.steps;
      s->completed += 1;
      s->group_dirty = true;
      it = s->trunning.erase(it);
      s->cv_done.notify_all();
    }
  }
}

}  // namespace

extern "C" {

int cep_serve_start(int model, int precision, int capacity, double dt, double dt_write, double max_bcl,
                    long steps_per_launch, double hbm_fraction, void *stream, cep_server_t *out) {
  if (!out) return cep_internal_set_fail(CEP_ERR_ARG, "out is NULL");
  *out = nullptr;
  if (!(dt > 0) || !(dt_write > 0) || !(max_bcl > 0) || steps_per_launch <= 0)
    return cep_internal_set_fail(CEP_ERR_ARG, "dt, dt_write, max_bcl and steps_per_launch must be positive");
  if (!(hbm_fraction > 0) || hbm_fraction > 1)
    return cep_internal_set_fail(CEP_ERR_ARG, "hbm_fraction must be in (0, 1]");
  if (cep_device_count() == 0) return cep_internal_set_fail(CEP_ERR_NO_DEVICE, "no CUDA device visible");
  // Ca samples per beat exactly as cep_batch_start_range counts them
  const int print_freq = (int)((1. / dt) * dt_write);
  const int per_beat = (print_freq > 0 ? (int)(max_bcl / dt) / print_freq : 0) + 2;
  // HBM admission: the pool may use hbm_fraction of the memory free now
  size_t free_b = 0, total_b = 0;
  if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess)
    return cep_internal_set_fail(CEP_ERR_CUDA, "cudaMemGetInfo failed");
  // states + parameters (<= 64 + 96 doubles), clock and schedule, biomarker
  // records, two Ca rings of per_beat + 2 doubles
  const double per_instance = 8.0 * (64 + 96 + 8 + 48 + 2.0 * (per_beat + 2)) + 64;
  const long long fit = (long long)(hbm_fraction * (double)free_b / per_instance);
  if (capacity <= 0) capacity = (int)std::min<long long>(fit, 1 << 24);
  if ((long long)capacity > fit) return cep_internal_set_fail(CEP_ERR_OOM, "capacity exceeds the HBM budget");
  if (capacity <= 0) return cep_internal_set_fail(CEP_ERR_OOM, "no room for a pool");
  cep_server *s = new cep_server;
  s->model = model;
  s->precision = precision;
  s->capacity = capacity;
  s->dt = dt;
  s->dt_write = dt_write;
  s->max_per_beat = per_beat;
  s->steps_per_launch = steps_per_launch;
  int rc;
  if ((rc = cep_batch_create(model, capacity, precision, stream, &s->pool)) ||
      (rc = cep_batch_init(s->pool, nullptr, nullptr, nullptr, 0, CEP_FLAG_QUIRKS)) ||
      (rc = cep_batch_reserve_biomarkers(s->pool, per_beat, dt, dt_write, -1e300))) {
    if (s->pool) cep_batch_destroy(s->pool);
    delete s;
    return rc;
  }
  s->owner.assign(capacity, -1);
  const double pool_bytes = per_instance * (double)capacity;
  const double budget = hbm_fraction * (double)free_b - pool_bytes;
  s->tissue_budget = budget > 0 ? (size_t)budget : 0;
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) == cudaSuccess && cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess)
    s->max_tissues = std::max(1, std::min(64, sms));
  if (cudaStreamCreateWithFlags(&s->tstream, cudaStreamNonBlocking) != cudaSuccess) {
    cep_batch_destroy(s->pool);
    delete s;
    return cep_internal_set_fail(CEP_ERR_CUDA, "stream for tissue jobs");
  }
  s->t_start = Clock::now();
  s->worker = std::thread(worker_loop, s);
  *out = s;
  return CEP_OK;
}

int cep_serve_submit(cep_server_t s, const cep_job_t *job, uint64_t *id) {
  if (!s || !job || !id) return cep_internal_set_fail(CEP_ERR_ARG, "null argument");
  if (job->n <= 0 || job->n > s->capacity) return cep_internal_set_fail(CEP_ERR_ARG, "job size outside 1..capacity");
  if (!job->conc) return cep_internal_set_fail(CEP_ERR_ARG, "conc is NULL");
  if (job->hill && job->hill_stride < 14) return cep_internal_set_fail(CEP_ERR_ARG, "hill_stride must be >= 14");
  if (!(job->bcl > 0) || job->n_pace <= 0 || job->first_pace >= job->n_pace)
    return cep_internal_set_fail(CEP_ERR_ARG, "bad protocol");
  const int print_freq = (int)((1. / s->dt) * s->dt_write);
  if (job->first_pace >= 0 && print_freq > 0 && (int)(job->bcl / s->dt) / print_freq + 2 > s->max_per_beat)
    return cep_internal_set_fail(CEP_ERR_ARG, "BCL longer than the server's max_bcl");
  auto j = std::make_shared<Job>();
  j->n = job->n;
  j->conc.assign(job->conc, job->conc + job->n);
  if (job->celltype) j->celltype.assign(job->celltype, job->celltype + job->n);
  if (job->hill) j->hill.assign(job->hill, job->hill + (size_t)job->n * job->hill_stride);
  j->hill_stride = job->hill ? job->hill_stride : 0;
  j->bcl = job->bcl;
  j->n_pace = job->n_pace;
  j->first_pace = job->first_pace;
  j->flags = job->flags;
  j->steps = (long long)job->n * (long long)((job->n_pace * job->bcl) / s->dt);
  j->t_submit = Clock::now();
  std::lock_guard<std::mutex> lock(s->mu);
  if (s->stop) return cep_internal_set_fail(s->fatal ? s->fatal : CEP_ERR_STATE, "server stopped");
  j->id = s->next_id++;
  s->jobs[j->id] = j;
  s->queue.push_back(j);
  *id = j->id;
  s->cv_work.notify_one();
  return CEP_OK;
}

int cep_serve_submit_tissue(cep_server_t s, const cep_tissue_job_t *job, uint64_t *id) {
  if (!s || !job || !id) return cep_internal_set_fail(CEP_ERR_ARG, "null argument");
  if (job->nx < 2 || job->ny < 2 || (long long)job->nx * job->ny > (1LL << 28))
    return fail_fmt(CEP_ERR_ARG, "patch of %d x %d nodes", job->nx, job->ny);
  if (!(job->h > 0) || !(job->D >= 0) || !(job->dt > 0) || !(job->duration > 0) || !(job->bcl > 0) || job->conc < 0)
    return cep_internal_set_fail(CEP_ERR_ARG, "h, dt, duration and bcl must be positive, D and conc >= 0");
  auto j = std::make_shared<Job>();
  j->tissue = true;
  j->tj = *job;
  j->tj.hill = nullptr;
  if (job->hill) j->thill.assign(job->hill, job->hill + 14);
  j->n = job->nx * job->ny;
  j->t_total = std::max(1L, (long)std::llround(job->duration / job->dt));
  j->steps = (long long)j->n * j->t_total;
  j->bytes = tissue_bytes(j->n);
  j->t_submit = Clock::now();
  std::lock_guard<std::mutex> lock(s->mu);
  if (s->stop) return cep_internal_set_fail(s->fatal ? s->fatal : CEP_ERR_STATE, "server stopped");
  if (j->bytes > s->tissue_budget)
    return fail_fmt(CEP_ERR_OOM, "patch needs %zu bytes, the tissue budget is %zu", j->bytes, s->tissue_budget);
  j->id = s->next_id++;
  s->jobs[j->id] = j;
  s->tqueue.push_back(j);
  *id = j->id;
  s->cv_work.notify_one();
  return CEP_OK;
}

int cep_serve_tissue_result(cep_server_t s, uint64_t id, double *v, double *t_act, cep_job_times_t *times) {
  if (!s) return cep_internal_set_fail(CEP_ERR_ARG, "null server");
  std::lock_guard<std::mutex> lock(s->mu);
  auto it = s->jobs.find(id);
  if (it == s->jobs.end()) return cep_internal_set_fail(CEP_ERR_ARG, "unknown job id");
  Job &j = *it->second;
  if (!j.tissue) return cep_internal_set_fail(CEP_ERR_ARG, "not a tissue job");
  if (j.state != CEP_JOB_DONE) return cep_internal_set_fail(CEP_ERR_STATE, "job not done");
  if (v) std::memcpy(v, j.v.data(), sizeof(double) * j.v.size());
  if (t_act) std::memcpy(t_act, j.tact.data(), sizeof(double) * j.tact.size());
  if (times) {
    times->queue_ms = ms_between(j.t_submit, j.t_admit);
    times->latency_ms = ms_between(j.t_submit, j.t_done);
    times->run_ms = ms_between(j.t_admit, j.t_done);
    times->cell_steps = (double)j.steps;
  }
  return CEP_OK;
}

int cep_serve_poll(cep_server_t s, uint64_t id, int *state) {
  if (!s || !state) return cep_internal_set_fail(CEP_ERR_ARG, "null argument");
  std::lock_guard<std::mutex> lock(s->mu);
  auto it = s->jobs.find(id);
  if (it == s->jobs.end()) return cep_internal_set_fail(CEP_ERR_ARG, "unknown job id");
  *state = it->second->state;
  return CEP_OK;
}

int cep_serve_wait(cep_server_t s, uint64_t id, double timeout_s) {
  if (!s) return cep_internal_set_fail(CEP_ERR_ARG, "null server");
  std::unique_lock<std::mutex> lock(s->mu);
  auto it = s->jobs.find(id);
  if (it == s->jobs.end()) return cep_internal_set_fail(CEP_ERR_ARG, "unknown job id");
  auto j = it->second;
  auto finished = [&] {
    return j->state == CEP_JOB_DONE || j->state == CEP_JOB_FAILED || j->state == CEP_JOB_CANCELLED;
  };
  if (timeout_s > 0) {
    if (!s->cv_done.wait_for(lock, std::chrono::duration<double>(timeout_s), finished))
      return cep_internal_set_fail(CEP_ERR_TIMEOUT, "job not finished within the timeout");
  } else {
    s->cv_done.wait(lock, finished);
  }
  if (j->state == CEP_JOB_FAILED)
    return fail_fmt(j->error ? j->error : CEP_ERR_STATE, "job failed: %s", j->msg.empty() ? "stopped" : j->msg.c_str());
  if (j->state == CEP_JOB_CANCELLED) return cep_internal_set_fail(CEP_ERR_STATE, "job cancelled");
  return CEP_OK;
}

int cep_serve_cancel(cep_server_t s, uint64_t id) {
  if (!s) return cep_internal_set_fail(CEP_ERR_ARG, "null server");
  std::lock_guard<std::mutex> lock(s->mu);
  auto it = s->jobs.find(id);
  if (it == s->jobs.end()) return cep_internal_set_fail(CEP_ERR_ARG, "unknown job id");
  auto j = it->second;
  if (j->state != CEP_JOB_QUEUED && j->state != CEP_JOB_RUNNING)
    return cep_internal_set_fail(CEP_ERR_STATE, "job already finished");
  for (auto *q : {&s->queue, &s->tqueue}) {
    auto pos = std::find(q->begin(), q->end(), j);
    if (pos != q->end()) {  // not admitted yet: it leaves at once
      q->erase(pos);
      j->t_admit = j->t_done = Clock::now();
      j->state = CEP_JOB_CANCELLED;
      s->cv_done.notify_all();
      return CEP_OK;
    }
  }
  j->cancel = true;  // admitted (or being admitted): the scheduler releases it between launches
  s->cv_work.notify_all();
  return CEP_OK;
}

int cep_serve_result(cep_server_t s, uint64_t id, cep_biomarkers_t *out, cep_job_times_t *times) {
  if (!s) return cep_internal_set_fail(CEP_ERR_ARG, "null server");
  std::lock_guard<std::mutex> lock(s->mu);
  auto it = s->jobs.find(id);
  if (it == s->jobs.end()) return cep_internal_set_fail(CEP_ERR_ARG, "unknown job id");
  Job &j = *it->second;
  if (j.state != CEP_JOB_DONE) return cep_internal_set_fail(CEP_ERR_STATE, "job not done");
  if (j.tissue) return cep_internal_set_fail(CEP_ERR_ARG, "a tissue job: use cep_serve_tissue_result");
  if (out) std::memcpy(out, j.result.data(), sizeof(cep_biomarkers_t) * j.n);
  if (times) {
    times->queue_ms = ms_between(j.t_submit, j.t_admit);
    times->latency_ms = ms_between(j.t_submit, j.t_done);
    times->run_ms = ms_between(j.t_admit, j.t_done);
    times->cell_steps = (double)j.steps;
  }
  return CEP_OK;
}

int cep_serve_release(cep_server_t s, uint64_t id) {
  if (!s) return cep_internal_set_fail(CEP_ERR_ARG, "null server");
  std::lock_guard<std::mutex> lock(s->mu);
  auto it = s->jobs.find(id);
  if (it == s->jobs.end()) return cep_internal_set_fail(CEP_ERR_ARG, "unknown job id");
  if (it->second->state != CEP_JOB_DONE && it->second->state != CEP_JOB_FAILED &&
      it->second->state != CEP_JOB_CANCELLED)
    return cep_internal_set_fail(CEP_ERR_STATE, "job still queued or running");
  s->jobs.erase(it);
  return CEP_OK;
}

int cep_serve_stats(cep_server_t s, cep_serve_stats_t *st) {
  if (!s || !st) return cep_internal_set_fail(CEP_ERR_ARG, "null argument");
  std::lock_guard<std::mutex> lock(s->mu);
  st->capacity = s->capacity;
  st->queued = (int)(s->queue.size() + s->tqueue.size());
  st->running = (int)(s->running.size() + s->trunning.size());
  int used = 0;
  for (int o : s->owner) used += o >= 0;
  st->slots_used = used;
  st->completed = s->completed;
  st->launches = s->launches;
  st->cell_steps = (double)s->steps_done;
  st->busy_ms = s->busy_ms;
  st->wall_ms = ms_between(s->t_start, Clock::now());
  return CEP_OK;
}

int cep_serve_stop(cep_server_t s) {
  if (!s) return CEP_OK;
  {
    std::lock_guard<std::mutex> lock(s->mu);
    s->stop = true;
    for (auto &j : s->queue) {
      j->state = CEP_JOB_FAILED;
      j->error = CEP_ERR_STATE;
    }
    for (auto &j : s->running) {
      j->state = CEP_JOB_FAILED;
      j->error = CEP_ERR_STATE;
    }
    for (auto &j : s->tqueue) {
      j->state = CEP_JOB_FAILED;
      j->error = CEP_ERR_STATE;
    }
    for (auto &j : s->trunning) {
      j->state = CEP_JOB_FAILED;
      j->error = CEP_ERR_STATE;
    }
    s->queue.clear();
    s->tqueue.clear();
  }
  s->cv_work.notify_all();
  s->cv_done.notify_all();
  if (s->worker.joinable()) s->worker.join();
  if (s->group) cep_tissue_group_destroy(s->group);
  for (auto &j : s->trunning) tissue_free(*j);
  s->trunning.clear();
  if (s->tstream) cudaStreamDestroy(s->tstream);
  cep_batch_destroy(s->pool);
  delete s;
  return CEP_OK;
}

}  // extern "C"
