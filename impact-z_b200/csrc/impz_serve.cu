// impz_serve.cu -- the serving loop: simulation jobs arriving over time share
// one GPU with continuous batching.
//
// A worker thread owns every device call.  Submitted jobs wait in a FIFO
// queue; a job is admitted as soon as its footprint (impz_bunch_footprint)
// fits the HBM budget next to the running jobs and a slot is free.  Each
// admitted job gets its own bunch and its state stays resident in HBM until
// it finishes.  The worker advances all running jobs of a form together in
// chunks of steps with packed launches (one launch per kernel for every job,
// each job at its own step of its own lattice), keeping at most two chunks in
// flight, so a job that arrives while others run joins them at the next
// chunk.  The actual device
// memory a job holds is measured at admission (cudaMemGetInfo before and
// after its bunch is created) and reported with the statistics.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <vector>

#include "../../include/impz_b200.h"

namespace {

using Clock = std::chrono::steady_clock;

struct Job {
  long long id = 0;
  // inputs (owned copies)
  std::vector<double> pts;
  long long n = 0;
  double current = 0, mass = 0, charge = 0, freq = 0;
  double refptcl[6] = {0};
  int nx = 0, ny = 0, nz = 0, form = 0;
  std::vector<impz_elem_t> elems;
  std::vector<std::vector<double>> tables;  // RF on-axis tables, 4 per element
  // state
  // 0 queued, 1 running, 2 done, <0 error code; written under the server
  // mutex, and set to 2 or an error only once the worker is done with the job
  int status = 0;
  int fin = 0;     // worker-private outcome: 0 running, 2 done, <0 error code
  impz_bunch_t bunch = nullptr;
  long long footprint = 0, measured = 0;
  int remaining = 0, chunks = 0;
  cudaEvent_t ev[2] = {nullptr, nullptr};
  Clock::time_point t_submit, t_start, t_done;
  // results
  std::vector<double> recs, zs;
  int nrec = 0;
  long long steps = 0;
};

}  // namespace

struct impz_server_s {
  int device = 0;
  double budget = 0;
  int max_active = 0;
  int chunk = 8;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<Job*> queue;
  std::vector<Job*> active;
  std::map<long long, Job*> jobs;
  long long next_id = 1;
  long long used = 0, peak_used = 0, peak_measured = 0;
  long long completed = 0, failed = 0;
  double particle_steps = 0;
  bool have_first = false;
  Clock::time_point t_first, t_last;
  bool stop = false;
  std::thread worker;
};

namespace {

double seconds(Clock::time_point a, Clock::time_point b) {
  return std::chrono::duration<double>(b - a).count();
}

// Creates the job's bunch and starts its run (worker thread).
int admit(impz_server_t s, Job* j) {
  size_t free0 = 0, total = 0, free1 = 0;
  cudaMemGetInfo(&free0, &total);
  int r = impz_bunch_create(j->pts.data(), j->n, j->current, j->mass, j->charge, j->freq,
                            j->refptcl, j->nx, j->ny, j->nz, j->form, 0, &j->bunch);
  if (r) return r;
  cudaMemGetInfo(&free1, &total);
  j->measured = free0 > free1 ? (long long)(free0 - free1) : 0;
  r = impz_run_begin(j->bunch, j->elems.data(), (int)j->elems.size());
  if (r) return r;
  j->remaining = impz_count_steps(j->elems.data(), (int)j->elems.size());
  j->steps = j->remaining;
  for (int k = 0; k < 2; k++)
    if (cudaEventCreateWithFlags(&j->ev[k], cudaEventDisableTiming) != cudaSuccess)
      return IMPZ_ERR_CUDA;
  std::vector<double>().swap(j->pts);  // the device holds the state now
  return IMPZ_OK;
}

void release(impz_server_t s, Job* j) {
  for (int k = 0; k < 2; k++)
    if (j->ev[k]) cudaEventDestroy(j->ev[k]);
  j->ev[0] = j->ev[1] = nullptr;
  if (j->bunch) impz_bunch_destroy(j->bunch);
  j->bunch = nullptr;
  std::lock_guard<std::mutex> g(s->mu);
  s->used -= j->footprint;
}

// One pass over the running jobs; returns true if anything was launched or
// finished (worker thread).  The stepping jobs of each form advance
// together, `chunk` steps per call, with packed launches
// (impz_run_advance_packed: one launch per kernel for all of them), at most
// two calls in flight; a job that arrives joins at the next call.
bool service(impz_server_t s, std::vector<Job*>& running) {
  bool progress = false;
  for (int form = 0; form < 2; form++) {
    std::vector<Job*> step;
    bool ready = true;
    for (Job* j : running) {
      if (j->fin != 0 || j->remaining <= 0 || j->form != form) continue;
      // chunk k of a job may go once its chunk k-2 is done
      if (j->chunks >= 2 && cudaEventQuery(j->ev[j->chunks & 1]) == cudaErrorNotReady)
        ready = false;
      step.push_back(j);
    }
    if (step.empty() || !ready) continue;
    std::vector<impz_bunch_t> bs(step.size());
    std::vector<int> left(step.size(), 0);
    for (size_t k = 0; k < step.size(); k++) bs[k] = step[k]->bunch;
    const int r = impz_run_advance_packed(bs.data(), (int)bs.size(), s->chunk, left.data());
    for (size_t k = 0; k < step.size(); k++) {
      Job* j = step[k];
      if (r) {
        j->fin = r;
        continue;
      }
      j->remaining = left[k];
      cudaEventRecord(j->ev[j->chunks & 1], (cudaStream_t)impz_bunch_stream(j->bunch));
      j->chunks++;
    }
    progress = true;
  }
  for (Job* j : running) {
    if (j->fin != 0) continue;
    if (j->remaining > 0) continue;
    if (cudaEventQuery(j->ev[(j->chunks - 1) & 1]) == cudaSuccess) {
      const int cap = (int)j->steps + 1;
      j->recs.assign((size_t)cap * IMPZ_MOMREC, 0.0);
      j->zs.assign(cap, 0.0);
      int r = impz_run_fetch(j->bunch, j->recs.data(), j->zs.data(), cap, &j->nrec);
      j->t_done = Clock::now();
      j->fin = r ? r : 2;
      progress = true;
    }
  }
  return progress;
}

void worker_main(impz_server_t s) {
  cudaSetDevice(s->device);
  std::vector<Job*> running;
  for (;;) {
    // admission (FIFO, by footprint and free slots)
    std::vector<Job*> admit_now;
    {
      std::unique_lock<std::mutex> lk(s->mu);
      if (s->stop && s->queue.empty() && running.empty()) break;
      while (!s->queue.empty() && (int)running.size() + (int)admit_now.size() < s->max_active) {
        Job* j = s->queue.front();
        if (s->used + j->footprint > (long long)s->budget && !(running.empty() && admit_now.empty()))
          break;
        s->queue.pop_front();
        s->used += j->footprint;
        s->peak_used = std::max(s->peak_used, s->used);
        admit_now.push_back(j);
      }
      if (running.empty() && admit_now.empty()) {
        s->cv_work.wait_for(lk, std::chrono::milliseconds(20));
        continue;
      }
    }
    for (Job* j : admit_now) {
      j->t_start = Clock::now();
      int r = admit(s, j);
      if (r) {
        j->t_done = Clock::now();
        release(s, j);
        std::lock_guard<std::mutex> g(s->mu);
        s->failed++;
        j->status = r;  // the waiter may free the job from here on
        s->cv_done.notify_all();
        continue;
      }
      running.push_back(j);
      std::lock_guard<std::mutex> g(s->mu);
      j->status = 1;
      s->peak_measured = std::max(s->peak_measured, j->measured);
    }
    const bool progress = service(s, running);
    // retire finished jobs
    std::vector<Job*> still;
    for (Job* j : running) {
      if (j->fin == 0) {
        still.push_back(j);
        continue;
      }
      release(s, j);
      std::lock_guard<std::mutex> g(s->mu);
      if (j->fin == 2) {
        s->completed++;
        s->particle_steps += (double)j->n * (double)j->steps;
        s->t_last = j->t_done;
      } else {
        s->failed++;
      }
      j->status = j->fin;  // the waiter may free the job from here on
      s->cv_done.notify_all();
    }
    running.swap(still);
    if (!progress) std::this_thread::sleep_for(std::chrono::microseconds(50));
  }
}

}  // namespace

extern "C" {

int impz_server_create(double hbm_budget_bytes, int max_active, impz_server_t* out) {
  if (!out || !(hbm_budget_bytes > 0) || max_active < 1) return IMPZ_ERR_ARG;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return IMPZ_ERR_NODEVICE;
  impz_server_t s = new impz_server_s();
  cudaGetDevice(&s->device);
  s->budget = hbm_budget_bytes;
  s->max_active = max_active;
  s->worker = std::thread(worker_main, s);
  *out = s;
  return IMPZ_OK;
}

int impz_server_submit(impz_server_t s, const double* pts, long long n, double current,
                       double mass, double charge, double freq, const double refptcl[6],
                       int nx, int ny, int nz, int form, const impz_elem_t* elems, int nelem,
                       long long* job) {
  if (!s || !pts || n < 1 || !refptcl || !elems || nelem < 1 || !job) return IMPZ_ERR_ARG;
  if (impz_count_steps(elems, nelem) < 1) return IMPZ_ERR_ARG;
  Job* j = new Job();
  j->pts.assign(pts, pts + 9 * n);
  j->n = n;
  j->current = current;
  j->mass = mass;
  j->charge = charge;
  j->freq = freq;
  std::memcpy(j->refptcl, refptcl, sizeof(j->refptcl));
  j->nx = nx; j->ny = ny; j->nz = nz; j->form = form;
  j->elems.assign(elems, elems + nelem);
  for (impz_elem_t& e : j->elems) {
    if (e.ndata > 0 && e.zdat && e.edat && e.epdat && e.eppdat) {
      const double* src[4] = {e.zdat, e.edat, e.epdat, e.eppdat};
      for (int k = 0; k < 4; k++) j->tables.emplace_back(src[k], src[k] + e.ndata);
      const size_t b0 = j->tables.size() - 4;
      e.zdat = j->tables[b0].data();
      e.edat = j->tables[b0 + 1].data();
      e.epdat = j->tables[b0 + 2].data();
      e.eppdat = j->tables[b0 + 3].data();
    } else {
      e.ndata = 0;
      e.zdat = e.edat = e.epdat = e.eppdat = nullptr;
    }
  }
  j->footprint = impz_bunch_footprint(n, nx, ny, nz, form, 0,
                                      impz_count_steps(j->elems.data(), (int)j->elems.size()));
  if (j->footprint < 0) {
    delete j;
    return IMPZ_ERR_ARG;
  }
  if ((double)j->footprint > s->budget) {
    delete j;
    return IMPZ_ERR_BUDGET;
  }
  j->t_submit = Clock::now();
  std::lock_guard<std::mutex> g(s->mu);
  if (s->stop) {
    delete j;
    return IMPZ_ERR_STATE;
  }
  j->id = s->next_id++;
  if (!s->have_first) {
    s->have_first = true;
    s->t_first = j->t_submit;
  }
  s->jobs[j->id] = j;
  s->queue.push_back(j);
  *job = j->id;
  s->cv_work.notify_one();
  return IMPZ_OK;
}

int impz_server_wait(impz_server_t s, long long job, double timeout_s, double* recs, int maxrec,
                     int* nrec, double times[3]) {
  if (!s) return IMPZ_ERR_ARG;
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->jobs.find(job);
  if (it == s->jobs.end()) return IMPZ_ERR_ARG;
  Job* j = it->second;
  auto done = [&] { return j->status == 2 || j->status < 0; };
  if (timeout_s < 0)
    s->cv_done.wait(lk, done);
  else if (!s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), done))
    return 1;  // still running
  if (j->status < 0) {
    const int r = j->status;
    s->jobs.erase(it);
    delete j;
    return r;
  }
  const int ncopy = std::min(j->nrec, std::max(maxrec, 0));
  if (recs && ncopy > 0)
    std::memcpy(recs, j->recs.data(), (size_t)ncopy * IMPZ_MOMREC * sizeof(double));
  if (nrec) *nrec = j->nrec;
  if (times) {
    times[0] = seconds(j->t_submit, j->t_done);  // latency
    times[1] = seconds(j->t_submit, j->t_start); // queueing
    times[2] = (double)j->measured;              // measured device bytes
  }
  s->jobs.erase(it);
  delete j;
  return IMPZ_OK;
}

int impz_server_stats(impz_server_t s, double out[8]) {
  if (!s || !out) return IMPZ_ERR_ARG;
  std::lock_guard<std::mutex> g(s->mu);
  out[0] = (double)s->completed;
  out[1] = (double)s->failed;
  out[2] = s->particle_steps;
  out[3] = s->have_first ? seconds(s->t_first, s->t_last) : 0.0;
  out[4] = (double)s->used;
  out[5] = (double)s->peak_used;
  out[6] = (double)s->peak_measured;
  out[7] = (double)s->queue.size();
  return IMPZ_OK;
}

int impz_server_destroy(impz_server_t s) {
  if (!s) return IMPZ_ERR_ARG;
  {
    std::lock_guard<std::mutex> g(s->mu);
    s->stop = true;
    s->cv_work.notify_all();
  }
  if (s->worker.joinable()) s->worker.join();
  for (auto& kv : s->jobs) delete kv.second;
  delete s;
  return IMPZ_OK;
}

}  // extern "C"
