// Job runtime: many grids on one GPU at once.
//
// The reference runs one grid per process (a module-level singleton,
// src/FastScape_ctx.f90:9-36; FastScape_Execute_Step, src/FastScape_api.f90:201-263).
// A batch runs a work table of independent grids ("jobs": grid, parameters,
// number of steps) on one device.  Worker threads each own a CUDA stream and
// run one job at a time through the handle API (set-up, parameter upload,
// `nsteps` continental steps, copy-out), so the steps of different jobs
// overlap on the GPU: a single grid's sweeps are bound by the length of its
// flow paths, not by the GPU's throughput, and other jobs fill the idle SMs.
//
// Admission is by device memory: a job is started only when its workspace
// (fsb_workspace_bytes) fits beside the jobs already running within the
// batch's budget; jobs start in submission order.  Arenas come from the
// stream-ordered allocator, so starting and finishing jobs never
// synchronises the device.  Every job's result is independent of what else
// runs: the kernels' arithmetic and their order are fixed per node.
#include <chrono>
#include <condition_variable>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include <cuda_runtime.h>

#include "fastscape_b200.h"
#include "fsb_kernels.cuh"

namespace {

double now_s() {
  using namespace std::chrono;
  return duration<double>(steady_clock::now().time_since_epoch()).count();
}

struct Job {
  fsb_job spec;
  long long id = 0;
  size_t bytes = 0;
  int status = 0;
  std::string msg;
  double t_submit = 0, t_start = 0, t_end = 0;
  bool done = false;
  bool waited = false;  // a thread is waiting for it (one waiter per job)
};

}  // namespace

struct fsb_batch {
  int device = 0;
  size_t budget = 0;
  size_t in_use = 0;
  int running = 0;
  bool stop = false;
  int nworkers = 0;  // set before the workers start
  long long next_id = 1;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<Job*> pending;
  std::unordered_map<long long, std::unique_ptr<Job>> jobs;
  std::vector<std::thread> workers;
};

namespace {

// Runs one job on `stream`; returns 0 or an error code with `msg` set.
int run_job(Job& j, cudaStream_t stream, int instances, std::string& msg) {
  const fsb_job& s = j.spec;
  fsb_ctx* h = nullptr;
  void* arena = nullptr;
  int rc = fsb_create(&h);
  if (rc != 0) { msg = fsb_last_error(); return rc; }
  // each call runs only while every earlier one has succeeded: after a
  // failure (say the job's arena could not be had) nothing more is set up,
  // allocated or run for this job
  auto step = [&](auto&& call) {
    if (rc != 0) return;
    const int r = call();
    if (r != 0) { rc = r; msg = fsb_last_error(); }
  };
  step([&] { return fsb_set_nx_ny(h, s.nx, s.ny); });
  step([&] { return fsb_set_stream(h, stream); });
  step([&] { return fsb_set_concurrency(h, instances); });
  size_t bytes = 0;
  step([&] { return fsb_workspace_bytes(h, &bytes); });
  if (rc == 0) {
    const cudaError_t e = cudaMallocAsync(&arena, bytes, stream);
    if (e != cudaSuccess) { rc = 1; msg = std::string("device memory for the job: ") + cudaGetErrorString(e); arena = nullptr; }
  }
  step([&] { return fsb_setup(h, arena, bytes); });
  step([&] { return fsb_set_xl_yl(h, s.xl, s.yl); });
  step([&] { return fsb_set_dt(h, s.dt); });
  step([&] { return fsb_init_h(h, s.h0, FSB_HOST); });
  step([&] {
    return fsb_set_erosional_parameters(h, s.kf, s.kfsed, s.m, s.n, s.kd, s.kdsed, s.g1, s.g2, s.p, FSB_HOST);
  });
  step([&] { return fsb_set_u(h, s.u, FSB_HOST); });
  if (s.precip) step([&] { return fsb_set_precip(h, s.precip, FSB_HOST); });
  step([&] { return fsb_set_bc(h, s.bc); });
  step([&] { return fsb_set_precision(h, s.precision); });
  step([&] { return fsb_execute_steps(h, s.nsteps); });
  if (s.h_out) step([&] { return fsb_copy_field(h, FSB_H, s.h_out, FSB_HOST); });
  if (s.a_out) step([&] { return fsb_copy_field(h, FSB_DRAINAGE_AREA, s.a_out, FSB_HOST); });
  if (s.etot_out) step([&] { return fsb_copy_field(h, FSB_TOTAL_EROSION, s.etot_out, FSB_HOST); });
  fsb_destroy(h);  // the arena is caller-owned: freed here, after the handle
  if (arena) cudaFreeAsync(arena, stream);
  const cudaError_t e = cudaStreamSynchronize(stream);
  if (rc == 0 && e != cudaSuccess) { rc = 1; msg = cudaGetErrorString(e); }
  return rc;
}

void worker_main(fsb_batch* b) {
  cudaSetDevice(b->device);
  cudaStream_t stream = nullptr;
  const cudaError_t se = cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking);
  for (;;) {
    Job* j = nullptr;
    {
      std::unique_lock<std::mutex> lk(b->mu);
      // the head job starts once its workspace fits beside the running jobs
      // (a job larger than the whole budget was refused at submission)
      b->cv_work.wait(lk, [&] {
        return b->stop || (!b->pending.empty() && b->in_use + b->pending.front()->bytes <= b->budget);
      });
      if (b->stop) break;  // set only once nothing is pending or running
      j = b->pending.front();
      b->pending.pop_front();
      b->in_use += j->bytes;
      ++b->running;
      j->t_start = now_s();
    }
    std::string msg;
    int rc = 0;
    if (se != cudaSuccess) { rc = 1; msg = std::string("worker stream: ") + cudaGetErrorString(se); }
    else rc = run_job(*j, stream, b->nworkers, msg);
    {
      std::lock_guard<std::mutex> lk(b->mu);
      j->t_end = now_s();
      j->status = rc;
      j->msg = msg;
      j->done = true;
      b->in_use -= j->bytes;
      --b->running;
    }
    b->cv_done.notify_all();
    b->cv_work.notify_all();
  }
  if (se == cudaSuccess) cudaStreamDestroy(stream);
}

}  // namespace

extern "C" {

int fsb_batch_create(fsb_batch** out, int device, int workers, size_t mem_budget) {
  if (!out) return fsb::report_error("fsb_batch_create: null output pointer");
  if (workers < 1 || workers > 256) return fsb::report_error("fsb_batch_create: workers must be in 1..256");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev)
    return fsb::report_error("fsb_batch_create: no such CUDA device");
  auto* b = new fsb_batch;
  b->device = device;
  if (mem_budget == 0) {  // default: 90% of the memory free now
    size_t fr = 0, tot = 0;
    cudaSetDevice(device);
    cudaMemGetInfo(&fr, &tot);
    mem_budget = fr / 10 * 9;
  }
  b->budget = mem_budget;
  {  // keep freed job arenas in the stream-ordered pool for the next jobs
    cudaSetDevice(device);
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
      unsigned long long keep = mem_budget;
      cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
  }
  b->nworkers = workers;
  for (int w = 0; w < workers; ++w) b->workers.emplace_back(worker_main, b);
  *out = b;
  return 0;
}

int fsb_batch_submit(fsb_batch* b, const fsb_job* job, long long* id) {
  if (!b || !job || !id) return fsb::report_error("fsb_batch_submit: null argument");
  const fsb_job& s = *job;
  if (s.nx < 3 || s.ny < 3) return fsb::report_error("fsb_batch_submit: nx and ny must be at least 3");
  if (s.nsteps < 0) return fsb::report_error("fsb_batch_submit: negative nsteps");
  if (!s.h0 || !s.kf || !s.kd || !s.u) return fsb::report_error("fsb_batch_submit: h0, kf, kd and u are required");
  fsb_ctx* h = nullptr;
  size_t bytes = 0;
  if (fsb_create(&h) != 0) return 1;
  int rc = fsb_set_nx_ny(h, s.nx, s.ny);
  if (rc == 0) rc = fsb_workspace_bytes(h, &bytes);
  fsb_destroy(h);
  if (rc != 0) return rc;
  auto j = std::make_unique<Job>();
  j->spec = s;
  j->bytes = bytes + (size_t(1) << 20);
  {
    std::lock_guard<std::mutex> lk(b->mu);
    if (j->bytes > b->budget)
      return fsb::report_error("fsb_batch_submit: the job needs " + std::to_string(j->bytes) +
                               " bytes of device memory, more than the batch's budget of " +
                               std::to_string(b->budget));
    j->id = b->next_id++;
    j->t_submit = now_s();
    *id = j->id;
    b->pending.push_back(j.get());
    b->jobs.emplace(j->id, std::move(j));
  }
  b->cv_work.notify_all();
  return 0;
}

int fsb_batch_wait(fsb_batch* b, long long id, int* status, double* times) {
  if (!b) return fsb::report_error("fsb_batch_wait: null batch");
  std::unique_lock<std::mutex> lk(b->mu);
  auto it = b->jobs.find(id);
  if (it == b->jobs.end()) return fsb::report_error("fsb_batch_wait: unknown job id " + std::to_string(id));
  Job* j = it->second.get();
  if (j->waited)  // the first waiter erases the job when it returns
    return fsb::report_error("fsb_batch_wait: job " + std::to_string(id) + " is already being waited for");
  j->waited = true;
  b->cv_done.wait(lk, [&] { return j->done; });
  if (status) *status = j->status;
  if (times) { times[0] = j->t_submit; times[1] = j->t_start; times[2] = j->t_end; }
  const int st = j->status;
  const std::string msg = j->msg;
  b->jobs.erase(it);
  lk.unlock();
  if (st != 0) return fsb::report_error("job " + std::to_string(id) + ": " + msg);
  return 0;
}

int fsb_batch_run(fsb_batch* b, const fsb_job* jobs, int njobs, int* status, double* times) {
  if (!b || (njobs > 0 && !jobs)) return fsb::report_error("fsb_batch_run: null argument");
  std::vector<long long> ids(njobs, -1);
  int first_err = 0;
  std::string first_msg;
  for (int k = 0; k < njobs; ++k) {
    if (fsb_batch_submit(b, &jobs[k], &ids[k]) != 0) {
      if (status) status[k] = 1;
      if (!first_err) { first_err = 1; first_msg = fsb_last_error(); }
    }
  }
  for (int k = 0; k < njobs; ++k) {
    if (ids[k] < 0) continue;
    int st = 0;
    const int rc = fsb_batch_wait(b, ids[k], &st, times ? times + 3 * k : nullptr);
    if (status) status[k] = st;
    if (rc != 0 && !first_err) { first_err = rc; first_msg = fsb_last_error(); }
  }
  if (first_err) return fsb::report_error(first_msg);
  return 0;
}

int fsb_batch_memory(fsb_batch* b, size_t* in_use, size_t* budget, int* running, int* pending) {
  if (!b) return fsb::report_error("fsb_batch_memory: null batch");
  std::lock_guard<std::mutex> lk(b->mu);
  if (in_use) *in_use = b->in_use;
  if (budget) *budget = b->budget;
  if (running) *running = b->running;
  if (pending) *pending = (int)b->pending.size();
  return 0;
}

int fsb_batch_destroy(fsb_batch* b) {
  if (!b) return 0;
  {
    std::unique_lock<std::mutex> lk(b->mu);
    // let every submitted job finish, then stop the workers
    b->cv_done.wait(lk, [&] { return b->pending.empty() && b->running == 0; });
    b->stop = true;
  }
  b->cv_work.notify_all();
  for (auto& t : b->workers) t.join();
  delete b;
  return 0;
}

}  // extern "C"
