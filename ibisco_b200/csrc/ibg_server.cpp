// Serving loop: simulation jobs of different sizes on one GPU with
// continuous batching.
//
// A job is a system after the reference's setup phase (an ibg_setup) and a
// number of steps.  Submissions go into a queue from any host thread.  One
// service thread owns the GPU work:
// - it admits queued jobs, in order, while the job-slot count and the device
//   memory budget allow (ibg_estimate_bytes before creation, then
//   ibg_device_bytes once created);
// - it keeps every admitted job's coordinates, lists and tables resident;
// - it steps all admitted jobs together as one batch (ibg_batch), tick by
//   tick, each to its own last step;
// - it retires finished jobs between ticks: their final state is copied to
//   host memory and their device memory is freed, which makes room for the
//   queue.
// Jobs that arrive while others are on the GPU therefore join the running
// batch at the next tick.  A job's result is bitwise the same alone and in
// any mix, because batched systems are computed exactly as single ones.
// Built on the public C ABI only (ibisco_gpu.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/ibisco_gpu.h"

namespace {

using Clock = std::chrono::steady_clock;

double seconds_since(Clock::time_point t0, Clock::time_point t) {
  return std::chrono::duration<double>(t - t0).count();
}

struct Job {
  long long id = 0;
  ibg_setup* setup = nullptr;
  int nsteps = 0;
  int natoms = 0, nitems = 0;
  std::vector<float> s0, v0;
  float box[3] = {0, 0, 0};
  long long est = 0, bytes = 0;
  ibg_ctx* ctx = nullptr;
  int state = IBG_JOB_QUEUED;
  int status = IBG_OK;
  std::string err;
  Clock::time_point t_submit, t_start, t_done;
  int steps_done = 0;
  std::vector<float> sxyz, vxyz;
  ibg_obs obs;
};

}  // namespace

struct ibg_server {
  int device = 0, precision = IBG_PREC_FP32_FIXED, max_jobs = 64, tick = 100;
  long long budget = 0;
  std::thread th;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  bool stop = false;
  std::deque<Job*> incoming;          // guarded by mu
  std::map<long long, Job*> jobs;     // guarded by mu
  long long next_id = 1;
  // owned by the service thread
  std::deque<Job*> queue;
  std::vector<Job*> active;
  ibg_batch* batch = nullptr;
  long long in_use = 0;
  // statistics, guarded by mu
  double gpu_ms = 0.0;
  long long atom_steps = 0, ticks = 0, batch_builds = 0;
  long long peak_active = 0;
  long long peak_bytes = 0;
};

namespace {

void set_state(ibg_server* S, Job* j, int state, int status, const std::string& err) {
  std::lock_guard<std::mutex> g(S->mu);
  j->state = state;
  j->status = status;
  j->err = err;
  if (state == IBG_JOB_DONE || state == IBG_JOB_FAILED) j->t_done = Clock::now();
  S->cv_done.notify_all();
}

void drop_batch(ibg_server* S) {
  if (S->batch) {
    ibg_batch_destroy(S->batch);
    S->batch = nullptr;
  }
}

void release(ibg_server* S, Job* j) {
  if (j->ctx) {
    ibg_destroy(j->ctx);
    j->ctx = nullptr;
  }
  S->in_use -= j->bytes;
  j->bytes = 0;
  if (j->setup) {
    ibg_setup_free(j->setup);
    j->setup = nullptr;
  }
}

// Admit queued jobs in order while slots and memory allow.  An idle GPU
// admits the next job whatever its size.
bool admit(ibg_server* S) {
  bool changed = false;
  while (!S->queue.empty() && (int)S->active.size() < S->max_jobs) {
    Job* j = S->queue.front();
    if (!S->active.empty() && S->in_use + j->est > S->budget) break;
    S->queue.pop_front();
    ibg_ctx* c = nullptr;
    int rc = ibg_create(ibg_setup_desc(j->setup), S->precision, &c);
    if (rc == IBG_OK) rc = ibg_set_state(c, j->s0.data(), j->v0.data(), j->box);
    if (rc != IBG_OK) {
      std::string m = c ? ibg_last_error(c) : "ibg_create failed";
      if (c) ibg_destroy(c);
      release(S, j);
      set_state(S, j, IBG_JOB_FAILED, rc, m);
      continue;
    }
    j->ctx = c;
    j->bytes = ibg_device_bytes(c);
    S->in_use += j->bytes;
    j->s0.clear();
    j->s0.shrink_to_fit();
    j->v0.clear();
    j->v0.shrink_to_fit();
    S->active.push_back(j);
    {
      std::lock_guard<std::mutex> g(S->mu);
      j->state = IBG_JOB_RUNNING;
      j->t_start = Clock::now();
      S->peak_active = std::max(S->peak_active, (long long)S->active.size());
      S->peak_bytes = std::max(S->peak_bytes, S->in_use);
    }
    changed = true;
  }
  return changed;
}

// One tick of the batch; retires the jobs that reached their last step.
void tick(ibg_server* S) {
  const int n = (int)S->active.size();
  std::vector<ibg_ctx*> ctxs(n);
  std::vector<int> last(n);
  for (int k = 0; k < n; ++k) {
    ctxs[k] = S->active[k]->ctx;
    last[k] = S->active[k]->nsteps;
  }
  if (!S->batch) {
    int rc = ibg_batch_create(ctxs.data(), n, &S->batch);
    if (rc != IBG_OK) {
      for (Job* j : S->active) {
        release(S, j);
        set_state(S, j, IBG_JOB_FAILED, rc, "ibg_batch_create failed");
      }
      S->active.clear();
      return;
    }
    std::lock_guard<std::mutex> g(S->mu);
    ++S->batch_builds;
  }
  std::vector<ibg_obs> obs(n);
  ibg_batch_run(S->batch, S->tick, last.data(), obs.data());
  double ms = 0;
  ibg_batch_get_timing(S->batch, &ms, nullptr);
  long long as = 0;
  for (int k = 0; k < n; ++k) {
    Job* j = S->active[k];
    as += (long long)j->natoms * std::max(0, obs[k].step - j->steps_done);
    j->steps_done = obs[k].step;
    j->obs = obs[k];
  }
  {
    std::lock_guard<std::mutex> g(S->mu);
    S->gpu_ms += ms;
    S->atom_steps += as;
    ++S->ticks;
  }
  // retire finished and failed jobs (the batch must go before its contexts)
  std::vector<Job*> keep;
  bool retire = false;
  for (Job* j : S->active)
    if (j->obs.status != IBG_OK || j->steps_done >= j->nsteps) retire = true;
  if (!retire) return;
  drop_batch(S);
  for (Job* j : S->active) {
    if (j->obs.status != IBG_OK) {
      std::string m = ibg_last_error(j->ctx);
      release(S, j);
      set_state(S, j, IBG_JOB_FAILED, j->obs.status, m);
    } else if (j->steps_done >= j->nsteps) {
      j->sxyz.resize(3 * (size_t)j->nitems);
      j->vxyz.resize(3 * (size_t)j->natoms);
      int rc = ibg_get_state(j->ctx, j->sxyz.data(), nullptr, j->vxyz.data(), nullptr);
      std::string m = rc ? ibg_last_error(j->ctx) : "";
      release(S, j);
      set_state(S, j, rc ? IBG_JOB_FAILED : IBG_JOB_DONE, rc, m);
    } else {
      keep.push_back(j);
    }
  }
  S->active.swap(keep);
}

void service(ibg_server* S) {
  cudaSetDevice(S->device);
  for (;;) {
    {
      std::unique_lock<std::mutex> lk(S->mu);
      if (S->stop) break;
      if (S->active.empty() && S->queue.empty() && S->incoming.empty())
        S->cv_work.wait(lk, [&] { return S->stop || !S->incoming.empty(); });
      if (S->stop) break;
      while (!S->incoming.empty()) {
        S->queue.push_back(S->incoming.front());
        S->incoming.pop_front();
      }
    }
    if (admit(S)) drop_batch(S);  // a new member: rebuild the batch
    if (!S->active.empty()) tick(S);
  }
  drop_batch(S);
  for (Job* j : S->active) {
    release(S, j);
    set_state(S, j, IBG_JOB_FAILED, IBG_E_INVALID, "server stopped");
  }
  S->active.clear();
  std::deque<Job*> rest;
  {
    std::lock_guard<std::mutex> g(S->mu);
    rest.swap(S->incoming);
  }
  for (Job* j : S->queue) rest.push_back(j);
  S->queue.clear();
  for (Job* j : rest) {
    release(S, j);
    set_state(S, j, IBG_JOB_FAILED, IBG_E_INVALID, "server stopped");
  }
}

double percentile(std::vector<double> v, double p) {
  if (v.empty()) return 0.0;
  std::sort(v.begin(), v.end());
  const double x = p * (double)(v.size() - 1);
  const size_t i = (size_t)x;
  const double f = x - (double)i;
  return i + 1 < v.size() ? v[i] * (1.0 - f) + v[i + 1] * f : v[i];
}

}  // namespace

extern "C" {

int ibg_server_create(int device, int precision, long long hbm_budget, int max_jobs, int tick_steps,
                      ibg_server** out) {
  if (!out || max_jobs <= 0 || tick_steps <= 0) return IBG_E_INVALID;
  if (precision != IBG_PREC_FP32_FIXED && precision != IBG_PREC_FP64_PLAIN) return IBG_E_INVALID;
  *out = nullptr;
  if (cudaSetDevice(device) != cudaSuccess) return IBG_E_CUDA;
  size_t free_b = 0, total_b = 0;
  if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) return IBG_E_CUDA;
  auto* S = new ibg_server;
  S->device = device;
  S->precision = precision;
  S->budget = hbm_budget > 0 ? hbm_budget : (long long)(0.8 * (double)free_b);
  S->max_jobs = max_jobs;
  S->tick = tick_steps;
  S->th = std::thread(service, S);
  *out = S;
  return IBG_OK;
}

int ibg_server_submit(ibg_server* S, ibg_setup* setup, int nsteps, long long* job) {
  if (!S || !setup || nsteps <= 0) return IBG_E_INVALID;
  const ibg_desc* d = ibg_setup_desc(setup);
  if (!d) return IBG_E_INVALID;
  auto* j = new Job;
  j->setup = setup;
  j->nsteps = nsteps;
  j->natoms = d->natoms;
  j->nitems = d->nitems;
  j->s0.resize(3 * (size_t)d->natoms);
  j->v0.resize(3 * (size_t)d->natoms);
  int rc = ibg_setup_initial_state(setup, j->s0.data(), j->v0.data(), j->box);
  if (rc != IBG_OK) {
    delete j;
    return rc;
  }
  j->est = ibg_estimate_bytes(d, S->precision, j->box);
  j->t_submit = Clock::now();
  {
    std::lock_guard<std::mutex> g(S->mu);
    if (S->stop) {
      delete j;
      return IBG_E_INVALID;
    }
    j->id = S->next_id++;
    S->jobs[j->id] = j;
    S->incoming.push_back(j);
  }
  S->cv_work.notify_one();
  if (job) *job = j->id;
  return IBG_OK;
}

int ibg_server_wait(ibg_server* S, long long job, double timeout_s) {
  if (!S) return IBG_E_INVALID;
  std::unique_lock<std::mutex> lk(S->mu);
  auto it = S->jobs.find(job);
  if (it == S->jobs.end()) return IBG_E_INVALID;
  Job* j = it->second;
  auto done = [&] { return j->state == IBG_JOB_DONE || j->state == IBG_JOB_FAILED; };
  if (timeout_s < 0) S->cv_done.wait(lk, done);
  else S->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), done);
  return j->state;
}

int ibg_server_drain(ibg_server* S, double timeout_s) {
  if (!S) return IBG_E_INVALID;
  std::unique_lock<std::mutex> lk(S->mu);
  auto all = [&] {
    for (auto& kv : S->jobs)
      if (kv.second->state != IBG_JOB_DONE && kv.second->state != IBG_JOB_FAILED) return false;
    return true;
  };
  bool ok = timeout_s < 0 ? (S->cv_done.wait(lk, all), true)
                          : S->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), all);
  return ok ? IBG_OK : IBG_E_TIMEOUT;
}

int ibg_server_result(ibg_server* S, long long job, float* sxyz, float* vxyz, ibg_obs* last_obs, double* times) {
  if (!S) return IBG_E_INVALID;
  std::lock_guard<std::mutex> g(S->mu);
  auto it = S->jobs.find(job);
  if (it == S->jobs.end()) return IBG_E_INVALID;
  Job* j = it->second;
  if (j->state == IBG_JOB_FAILED) return j->status ? j->status : IBG_E_INVALID;
  if (j->state != IBG_JOB_DONE) return IBG_E_INVALID;
  if (sxyz) std::memcpy(sxyz, j->sxyz.data(), sizeof(float) * j->sxyz.size());
  if (vxyz) std::memcpy(vxyz, j->vxyz.data(), sizeof(float) * j->vxyz.size());
  if (last_obs) *last_obs = j->obs;
  if (times) {
    times[0] = seconds_since(j->t_submit, j->t_start);  // queued
    times[1] = seconds_since(j->t_start, j->t_done);    // admitted to done
    times[2] = seconds_since(j->t_submit, j->t_done);   // latency
  }
  return IBG_OK;
}

const char* ibg_server_job_error(ibg_server* S, long long job) {
  if (!S) return "null server";
  std::lock_guard<std::mutex> g(S->mu);
  auto it = S->jobs.find(job);
  return it == S->jobs.end() ? "unknown job" : it->second->err.c_str();
}

int ibg_server_get_stats(ibg_server* S, ibg_server_stats* out) {
  if (!S || !out) return IBG_E_INVALID;
  std::lock_guard<std::mutex> g(S->mu);
  std::memset(out, 0, sizeof(*out));
  std::vector<double> lat;
  bool any = false;
  Clock::time_point first{}, lastd{};
  for (auto& kv : S->jobs) {
    const Job* j = kv.second;
    ++out->submitted;
    if (!any || j->t_submit < first) first = j->t_submit;
    any = true;
    if (j->state == IBG_JOB_DONE) {
      ++out->done;
      lat.push_back(seconds_since(j->t_submit, j->t_done));
      if (j->t_done > lastd) lastd = j->t_done;
    } else if (j->state == IBG_JOB_FAILED) {
      ++out->failed;
    } else if (j->state == IBG_JOB_RUNNING) {
      ++out->running;
    } else {
      ++out->queued;
    }
  }
  out->p50_s = percentile(lat, 0.50);
  out->p99_s = percentile(lat, 0.99);
  out->mean_s = lat.empty() ? 0.0 : [&] { double s = 0; for (double x : lat) s += x; return s / lat.size(); }();
  const double span = out->done ? seconds_since(first, lastd) : 0.0;
  out->span_s = span;
  out->jobs_per_s = span > 0 ? (double)out->done / span : 0.0;
  out->atom_steps = S->atom_steps;
  out->atom_steps_per_s = span > 0 ? (double)S->atom_steps / span : 0.0;
  out->gpu_s = S->gpu_ms / 1000.0;
  out->ticks = S->ticks;
  out->batch_builds = S->batch_builds;
  out->peak_jobs = S->peak_active;
  out->peak_bytes = S->peak_bytes;
  out->budget_bytes = S->budget;
  return IBG_OK;
}

void ibg_server_destroy(ibg_server* S) {
  if (!S) return;
  {
    std::lock_guard<std::mutex> g(S->mu);
    S->stop = true;
  }
  S->cv_work.notify_all();
  if (S->th.joinable()) S->th.join();
  for (auto& kv : S->jobs) delete kv.second;
  delete S;
}

}  // extern "C"
